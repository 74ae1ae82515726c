"""Batched instances (ts_batch_*): one persistent launch per RK4 stage over all instances.

Each instance of a batch must give bitwise the same state as its own single-box integrator
(ts_integrator_*) on the same input: the batch runs the same fused stage kernels, only the
work distribution differs. The FP64 form is also checked against the CPU oracle
(<= 1e-12 relative max-norm), graph replays against eager launches, and the autotuner for
leaving the states untouched.
"""
import numpy as np
import pytest

import treesap_b200 as tsb
from treesap_b200 import TS_BC_DIRICHLET, TS_F32_STAGE, TS_F64, TS_INIT_GAUSSIAN, Batch, Integrator, TSError
from treesap_b200.configs import wave_desc

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def pulse(seed):
    rng = np.random.default_rng(seed)
    return np.array([[0, rng.uniform(0.5, 1.0), rng.uniform(0.05, 0.2), *rng.uniform(0.3, 0.7, 3)]])


def batch_descs(sizes, ngrow, precision, periodic=True, ko=0.0, bc_values=(0.0, 0.0)):
    out = []
    for n in sizes:
        n3 = (n, n, n) if np.isscalar(n) else tuple(n)
        per = (1, 1, 1) if periodic else (0, 0, 0)
        out.append(wave_desc(n3, ngrow, periodic=per, ko=ko, precision=precision, dt=0.25 / n3[0],
                             bc=TS_BC_NOOP_OR_DIRICHLET(periodic), bc_values=bc_values))
    return out


def TS_BC_NOOP_OR_DIRICHLET(periodic):
    return tsb.TS_BC_NOOP if periodic else TS_BC_DIRICHLET


SIZES = [16, (24, 20, 28), 40, (33, 17, 21), 48, (64, 8, 40)]


@pytest.mark.parametrize("precision", [TS_F64, TS_F32_STAGE])
@pytest.mark.parametrize("ngrow,ko,periodic", [(2, 0.0, True), (4, 0.2, False), (2, 0.1, False), (4, 0.0, True)])
def test_batch_matches_single_box_bitwise(ctx, precision, ngrow, ko, periodic):
    sizes = [s for s in SIZES if min(np.atleast_1d(s)) >= 2 * ngrow]
    descs = batch_descs(sizes, ngrow, precision, periodic=periodic, ko=ko, bc_values=(0.25, -0.5))
    b = Batch(ctx, descs)
    for i in range(len(descs)):
        b.initialise(i, TS_INIT_GAUSSIAN, pulse(i))
    b.step(3)
    b.step(2)
    ctx.sync()
    for i, d in enumerate(descs):
        it = Integrator(ctx, d)
        it.initialise(TS_INIT_GAUSSIAN, pulse(i))
        it.step(5)
        want = it.get_state()
        got = b.get_state(i)
        assert np.array_equal(got, want), (i, relerr(got, want))


@pytest.mark.parametrize("precision", [TS_F64, TS_F32_STAGE])
def test_batch_mixed_periodicity_matches_single_box_bitwise(ctx, precision):
    """Instances periodic in different directions (Dirichlet data on their other faces) in one
    batch: the batched ghost fill resolves periodic images and boundary cells per instance, and
    a thread's cells mix both kinds at the edges and corners of the faces."""
    shapes = [((24, 20, 28), (1, 0, 0)), ((33, 17, 21), (0, 1, 1)), ((16, 16, 16), (1, 1, 1)),
              ((40, 24, 16), (0, 0, 1)), ((20, 20, 20), (0, 0, 0)), ((18, 30, 12), (1, 1, 0))]
    descs = [wave_desc(n3, 2, periodic=per, ko=0.1, precision=precision, dt=0.25 / n3[0], bc=TS_BC_DIRICHLET,
                       bc_values=(0.25, -0.5)) for n3, per in shapes]
    b = Batch(ctx, descs)
    for i in range(len(descs)):
        b.initialise(i, TS_INIT_GAUSSIAN, pulse(i))
    b.step(4)
    ctx.sync()
    for i, d in enumerate(descs):
        it = Integrator(ctx, d)
        it.initialise(TS_INIT_GAUSSIAN, pulse(i))
        it.step(4)
        want = it.get_state()
        got = b.get_state(i)
        assert np.array_equal(got, want), (i, shapes[i], relerr(got, want))
    b.close()


def test_batch_fp64_matches_oracle(ctx, port_oracle):
    descs = batch_descs([20, (28, 16, 24)], 2, TS_F64, periodic=True, ko=0.1)
    b = Batch(ctx, descs)
    rng = np.random.default_rng(3)
    states = [rng.standard_normal(d.shape()) for d in descs]
    for i, s in enumerate(states):
        b.set_state(i, s)
    b.step(4)
    for i, d in enumerate(descs):
        cpu, _, _ = port_oracle.run(d, 4, state=states[i])
        assert relerr(b.get_state(i), cpu) <= TOL_F64


@pytest.mark.parametrize("periodic", [True, False])
def test_batch_graph_replay_is_bitwise_identical(ctx, periodic):
    descs = batch_descs([24, 32, (40, 24, 16)], 2, TS_F32_STAGE, periodic=periodic, ko=0.1)
    res = []
    for graph in (False, True):
        b = Batch(ctx, descs)
        for i in range(len(descs)):
            b.initialise(i, TS_INIT_GAUSSIAN, pulse(10 + i))
        b.use_graph(graph)
        for _ in range(5):
            b.step(1)
        b.step(3)
        ctx.sync()
        res.append([b.get_state(i) for i in range(len(descs))])
    for a, g in zip(*res):
        assert np.array_equal(a, g)


def test_batch_launch_counts(ctx):
    """One launch per stage and per ghost fill for the whole batch; static ghosts filled once."""
    periodic = Batch(ctx, batch_descs([16, 24, 32], 2, TS_F32_STAGE, periodic=True))
    periodic.step(2)
    ctx.sync()
    assert periodic.last_step_timing()[1] == 2 * 8
    fixed = Batch(ctx, batch_descs([16, 24, 32], 2, TS_F32_STAGE, periodic=False))
    fixed.step(2)
    fixed.step(2)
    ctx.sync()
    assert fixed.last_step_timing()[1] == 2 * 4


def test_batch_autotune_keeps_states(ctx):
    descs = batch_descs([16, 32, 48, (24, 40, 56)], 2, TS_F32_STAGE, periodic=True)
    ref = Batch(ctx, descs)
    tuned = Batch(ctx, descs)
    for b in (ref, tuned):
        for i in range(len(descs)):
            b.initialise(i, TS_INIT_GAUSSIAN, pulse(20 + i))
        b.step(2)
    rows, zchunk = tuned.autotune(2)
    assert 1 <= rows <= 7 and zchunk >= 0
    for b in (ref, tuned):
        b.step(3)
    ctx.sync()
    for i in range(len(descs)):
        assert np.array_equal(tuned.get_state(i), ref.get_state(i))


def test_batch_rejects_mixed_or_unsupported(ctx):
    a = wave_desc(16, 2)
    b = wave_desc(16, 4)
    with pytest.raises(TSError) as e:
        Batch(ctx, [a, b])
    assert e.value.status == 1
    abl = wave_desc(32, 2, periodic=(0, 0, 0), abl_thickness=4, abl_max=1.0, bc=TS_BC_DIRICHLET)
    with pytest.raises(TSError) as e:
        Batch(ctx, [abl])
    assert e.value.status == 2
