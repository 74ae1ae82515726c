"""FunctionInit expressions (init/FunctionInit.hpp, util/expression.hpp), checked on the host.

The library compiles an expression of x, y, z into a postfix program that the device
evaluates in the init kernel; ts_expression_eval runs the same program on the host. Here the
programs are compared with numpy on random points, invalid text must be refused, and the
reference's own example drivers (which initialise through FunctionInit) must compile unchanged.
"""
import math
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest
from scipy.special import erf

from treesap_b200 import TSError, expression_eval

ROOT = Path(__file__).resolve().parents[1]
from conftest import REFERENCE_SKIP, reference_root  # noqa: E402

REF = reference_root()

rng = np.random.default_rng(123)
X, Y, Z = rng.uniform(-1.0, 1.0, (3, 200))

CASES = [
    ("exp(-(x^2 + y^2 + z^2)/0.1^2)", lambda x, y, z: np.exp(-(x**2 + y**2 + z**2) / 0.1**2)),
    ("2^3^2 + x", lambda x, y, z: 512.0 + x),
    ("-x^2", lambda x, y, z: -(x**2)),
    ("2^-1 * y", lambda x, y, z: 0.5 * y),
    ("sin(pi*x)*cos(2*pi*y) + z", lambda x, y, z: np.sin(np.pi * x) * np.cos(2 * np.pi * y) + z),
    ("if(x < 0.25, 1, 2) + 0*y", lambda x, y, z: np.where(x < 0.25, 1.0, 2.0)),
    ("max(x, y) - min(y, z)", lambda x, y, z: np.maximum(x, y) - np.minimum(y, z)),
    ("atan2(y, x) + atan(z)", lambda x, y, z: np.arctan2(y, x) + np.arctan(z)),
    ("sqrt(abs(x - y)) + fabs(z)", lambda x, y, z: np.sqrt(np.abs(x - y)) + np.abs(z)),
    ("1e-3*x + .5 - 2.5E+1*z", lambda x, y, z: 1e-3 * x + 0.5 - 25.0 * z),
    ("x**2*y", lambda x, y, z: x**2 * y),
    ("(x > 0.2) and (y < 0.7) or z > 0.9", lambda x, y, z: (((x > 0.2) & (y < 0.7)) | (z > 0.9)).astype(float)),
    ("(x >= y) + (x <= z) + (x == x) + (y != y)", lambda x, y, z: (x >= y).astype(float) + (x <= z).astype(float) + 1.0),
    ("heaviside(x - 0.5) * 3", lambda x, y, z: np.where(x - 0.5 > 0, 3.0, 0.0)),
    ("fmod(x*7, 2)", lambda x, y, z: np.fmod(x * 7, 2)),
    ("floor(x*10)/10 + ceil(y)", lambda x, y, z: np.floor(x * 10) / 10 + np.ceil(y)),
    ("log(2 + x) + log10(2 + y)", lambda x, y, z: np.log(2 + x) + np.log10(2 + y)),
    ("tanh(x) + sinh(y) - cosh(z)", lambda x, y, z: np.tanh(x) + np.sinh(y) - np.cosh(z)),
    ("asin(x/2) + acos(y/2) + tan(z)", lambda x, y, z: np.arcsin(x / 2) + np.arccos(y / 2) + np.tan(z)),
    ("erf(x) + pow(abs(y), 1.5)", lambda x, y, z: erf(x) + np.abs(y) ** 1.5),
    ("0.0", lambda x, y, z: np.zeros_like(x)),
    ("  ( ( x ) )  ", lambda x, y, z: x),
]


@pytest.mark.parametrize("text,ref", CASES, ids=[c[0] for c in CASES])
def test_expression_matches_numpy(text, ref):
    got = expression_eval(text, X, Y, Z)
    want = ref(X, Y, Z)
    np.testing.assert_allclose(got, want, rtol=1e-14, atol=1e-14)


@pytest.mark.parametrize("text", ["exp(", "x +", "foo(x)", "2x", "((x)", "pow(x)", "x ** ", "if(x, 1)", "", "y $ 2"])
def test_invalid_expressions_are_refused(text):
    with pytest.raises(TSError) as e:
        expression_eval(text, X[:3], Y[:3], Z[:3])
    assert e.value.status == 1


@pytest.mark.skipif(REF is None, reason=REFERENCE_SKIP)
@pytest.mark.parametrize("example", ["examples/01-wave-eqn/main.cpp", "examples/02-temporaries/main.cpp"])
def test_reference_example_driver_compiles_unchanged(tmp_path, example):
    """The reference's example programs (FunctionInit, PDEModel, RK4 integrator, exporter,
    ScopedTimer) compile unchanged for sm_100a against these headers."""
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    src = REF / example
    inc = ["-I", str(ROOT / "include"), "-I", str(ROOT / "treesap_b200/cpp/compat"), "-I",
           str(ROOT / "treesap_b200/cpp/treesap"), "-I", str(src.parent)]
    cmd = [nvcc, "-std=c++20", "--expt-relaxed-constexpr", "--extended-lambda", "-gencode",
           "arch=compute_100a,code=sm_100a", *inc, "-x", "cu", "-c", str(src), "-o", str(tmp_path / "main.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
