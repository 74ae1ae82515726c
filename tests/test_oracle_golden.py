"""The CPU restatement (oracle/ts_oracle.c) against the reference's own results (tests/golden/).

Both are compiled without FMA contraction and follow the same operation order, so the
comparison is exact. Where the reference build exists (this container), it is also re-run
and must reproduce its fixtures bit for bit.
"""
import numpy as np
import pytest

from golden_cases import load, names, ref_desc, run_kwargs


@pytest.mark.parametrize("name", names())
def test_port_reproduces_reference_golden(port_oracle, name):
    d, inp, nsteps, t, out = load(name)
    got, _, tt = port_oracle.run(ref_desc(d), nsteps, **run_kwargs(inp))
    assert np.array_equal(got, out), float(np.abs(got - out).max())
    assert tt == t


@pytest.mark.parametrize("name", names())
def test_reference_build_reproduces_golden(name):
    from oracle import pyoracle

    if not pyoracle.available("ref"):
        pytest.skip("reference build not present")
    d, inp, nsteps, t, out = load(name)
    got, _, _ = pyoracle.Oracle("ref").run(ref_desc(d), nsteps, **run_kwargs(inp))
    assert np.array_equal(got, out)


def test_goldens_exist():
    assert len(names()) >= 15
