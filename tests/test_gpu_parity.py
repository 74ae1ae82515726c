"""Parity of the B200 kernels with the CPU oracle (FP64 plain form: <= 1e-12 relative max-norm).

Every case calls the library through the C ABI (ts_integrator_*) and runs the same seeded
input through the oracle (the reference's own integrators built on the host, or the
bit-identical plain-C restatement). Relative max-norm = max|gpu - cpu| / max|cpu|.
"""
import itertools

import numpy as np
import pytest

from treesap_b200 import (TS_BC_DIRICHLET, TS_BC_NOOP, TS_EULER, TS_F32_STAGE, TS_F64, TS_INIT_GAUSSIAN, TS_RK4,
                          Integrator)
from treesap_b200.configs import C1_STEPS, c1_desc, c1_pulses, c2_pulses, wave_desc

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-12  # FP64 plain form vs oracle, relative max-norm


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def smooth_state(shape, seed):
    """Seeded smooth-ish random state (sum of a few low Fourier modes plus small noise)."""
    rng = np.random.default_rng(seed)
    nc, nz, ny, nx = shape
    z, y, x = np.meshgrid(np.arange(nz) / nz, np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")
    s = np.zeros(shape)
    for c in range(nc):
        for _ in range(4):
            k = rng.integers(-2, 3, 3)
            s[c] += rng.normal() * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + rng.uniform(0, 6.28))
        s[c] += 0.01 * rng.standard_normal((nz, ny, nx))
    return s


CASES = list(itertools.product([1, 2, 3, 4], ["periodic", "dirichlet", "abl"], [0.0, 0.15], [TS_RK4, TS_EULER]))


@pytest.mark.parametrize("ngrow,bcmode,ko,scheme", CASES)
def test_fp64_matches_oracle_small(ctx, port_oracle, ngrow, bcmode, ko, scheme):
    n = (37, 29, 41)  # partial tiles in x, y and uneven z segments
    kw = dict(prob_lo=(-1.0, 0.0, 0.5), prob_hi=(1.0, 1.0, 2.0), ko=ko, scheme=scheme, dt=0.2 / 41)
    if bcmode == "periodic":
        d = wave_desc(n, ngrow, periodic=(1, 1, 1), **kw)
    elif bcmode == "dirichlet":
        d = wave_desc(n, ngrow, periodic=(1, 0, 0), bc=TS_BC_DIRICHLET, bc_values=(0.3, -0.2), **kw)
    else:
        d = wave_desc(n, ngrow, periodic=(0, 0, 0), abl_thickness=5, abl_max=7.0, abl_profile=2,
                      bc=TS_BC_DIRICHLET, bc_values=(0.1, 0.0), **kw)
    state = smooth_state(d.shape(), seed=ngrow * 100 + int(ko * 100) + scheme)
    it = Integrator(ctx, d)
    it.set_state(state)
    it.step(4)
    gpu = it.get_state()
    ctx.sync()
    cpu, _, tcpu = port_oracle.run(d, 4, state=state)
    assert relerr(gpu, cpu) <= TOL_F64
    t, s = it.time()
    assert s == 4 and abs(t - tcpu) == 0.0


def test_c1_full_run_matches_oracle(ctx, oracle):
    """C1: 64^3 periodic, ngrow 2, KO 0.1, RK4, 100 steps from the Gaussian initialiser."""
    d = c1_desc()
    it = Integrator(ctx, d)
    it.initialise(TS_INIT_GAUSSIAN, c1_pulses())
    it.step(C1_STEPS)
    gpu = it.get_state()
    ctx.sync()
    cpu, _, _ = oracle.run(d, C1_STEPS, items=c1_pulses())
    assert relerr(gpu, cpu) <= TOL_F64


def test_initialise_matches_oracle(ctx, port_oracle):
    d = wave_desc((33, 20, 27), 3, periodic=(0, 1, 0), bc=TS_BC_DIRICHLET)
    pul = c2_pulses(7, 5)
    pul[2, 0] = 1  # one pulse on pi
    it = Integrator(ctx, d)
    it.initialise(TS_INIT_GAUSSIAN, pul)
    gpu = it.get_state()
    cpu, _, _ = port_oracle.run(d, 0, items=pul)
    assert relerr(gpu, cpu) <= 1e-14


def test_state_roundtrip_is_exact(ctx):
    d = wave_desc((19, 23, 17), 4, periodic=(0, 0, 1))
    s = smooth_state(d.shape(), 3)
    it = Integrator(ctx, d)
    it.set_state(s)
    assert np.array_equal(it.get_state(), s)


def test_graph_replay_is_bitwise_identical(ctx):
    d = wave_desc(48, 2, ko=0.1)
    s = smooth_state(d.shape(), 5)
    a = Integrator(ctx, d)
    a.set_state(s)
    a.step(7)
    ra = a.get_state()
    b = Integrator(ctx, d)
    b.use_graph(True)
    b.set_state(s)
    b.step(3)
    b.step(4)
    rb = b.get_state()
    assert np.array_equal(ra, rb)
    assert b.time()[1] == 7


def test_variable_speed_matches_oracle(ctx, port_oracle):
    d = wave_desc(32, 2, ko=0.1)
    rng = np.random.default_rng(11)
    c2 = (1.0 + 0.2 * rng.uniform(-1, 1, (32, 32, 32))) ** 2
    s = smooth_state(d.shape(), 9)
    it = Integrator(ctx, d, c2=c2)
    it.set_state(s)
    it.step(5)
    gpu = it.get_state()
    cpu, _, _ = port_oracle.run(d, 5, state=s, c2=c2)
    assert relerr(gpu, cpu) <= TOL_F64


@pytest.mark.parametrize("ngrow,periodic", [(2, (1, 1, 1)), (4, (0, 0, 0)), (3, (1, 0, 1))])
def test_fp32_stage_without_decorators(ctx, ngrow, periodic):
    """FP32-stage RK4 of the undecorated wave model (no Kreiss-Oliger, no layer): the right-hand
    side is its own linear part, so stages 0 and 1 run the same functor type."""
    bc = TS_BC_NOOP if all(periodic) else TS_BC_DIRICHLET
    mk = lambda p: wave_desc((40, 36, 32), ngrow, periodic=periodic, bc=bc, precision=p, dt=0.25 / 40)
    pul = c2_pulses(1, 4)
    out = {}
    for p in (TS_F64, TS_F32_STAGE):
        it = Integrator(ctx, mk(p))
        it.initialise(TS_INIT_GAUSSIAN, pul)
        it.step(40)
        out[p] = it.get_state()
    ctx.sync()
    assert np.abs(out[TS_F64]).max() > 0.1
    assert relerr(out[TS_F32_STAGE], out[TS_F64]) <= 1e-6


@pytest.mark.parametrize("bcmode", ["periodic", "abl"])
def test_fp32_stage_error_vs_fp64(ctx, bcmode):
    """FP32-stage RK4 vs FP64 GPU path: max-norm relative error <= 1e-6 after 200 steps."""
    if bcmode == "periodic":
        mk = lambda p: wave_desc(64, 4, ko=0.2, precision=p)
    else:
        mk = lambda p: wave_desc(64, 4, periodic=(0, 0, 0), ko=0.2, abl_thickness=8, abl_max=10.0,
                                 bc=TS_BC_DIRICHLET, precision=p)
    pul = c2_pulses(1, 4)
    out = {}
    for p in (TS_F64, TS_F32_STAGE):
        it = Integrator(ctx, mk(p))
        it.initialise(TS_INIT_GAUSSIAN, pul)
        it.step(200)
        out[p] = it.get_state()
    ctx.sync()
    e = relerr(out[TS_F32_STAGE], out[TS_F64])
    assert e <= 1e-6, e


@pytest.mark.parametrize("precision", [TS_F64, TS_F32_STAGE])
def test_static_ghost_fills_run_once_per_buffer(ctx, port_oracle, precision):
    """Non-periodic Dirichlet data: each buffer's ghost cells are filled once, later fills skipped.

    RK4 FP64: step 1 fills u, arg (twice: two stage buffers) = 3 fills + 4 stages; step 2 fills
    the other state buffer = 1 + 4; from step 3 on only the 4 stage kernels run. A periodic
    direction keeps every fill (4 + 4). The results still match the oracle.
    """
    n = (36, 30, 34)
    mk = lambda periodic: wave_desc(n, 2, periodic=periodic, ko=0.1, bc=TS_BC_DIRICHLET, bc_values=(0.0, 0.0),
                                    precision=precision, dt=0.2 / 36)
    state = smooth_state((2, n[2], n[1], n[0]), seed=5)
    d = mk((0, 0, 0))
    it = Integrator(ctx, d)
    it.set_state(state)
    counts = []
    for _ in range(4):
        it.step(1)
        ctx.sync()
        counts.append(it.last_step_timing()[1])
    want = [7, 5, 4, 4] if precision == TS_F64 else [4 + 4, 4 + 1, 4, 4]
    assert counts == want, counts
    gpu = it.get_state()
    if precision == TS_F64:
        cpu, _, _ = port_oracle.run(d, 4, state=state)
        assert relerr(gpu, cpu) <= TOL_F64
    it_p = Integrator(ctx, mk((1, 0, 0)))
    it_p.set_state(state)
    it_p.step(1)
    it_p.step(1)
    ctx.sync()
    assert it_p.last_step_timing()[1] == 8


def test_function_init_expressions_match_numpy(ctx):
    """FunctionInit through the C ABI: device evaluation of the compiled expressions at cell centres."""
    n = (20, 24, 28)
    lo, hi = (-2.0, -1.0, 0.0), (2.0, 1.0, 1.5)
    d = wave_desc(n, 2, periodic=(0, 0, 0), prob_lo=lo, prob_hi=hi, bc=TS_BC_DIRICHLET)
    it = Integrator(ctx, d)
    it.initialise_expressions(["exp(-(x^2 + y^2 + z^2)/0.5^2)", "sin(pi*x)*y + z^3 - if(x < 0, 1, 0)"])
    got = it.get_state()
    c = [lo[a] + (np.arange(n[a]) + 0.5) * (hi[a] - lo[a]) / n[a] for a in range(3)]
    z, y, x = np.meshgrid(c[2], c[1], c[0], indexing="ij")
    want = np.stack([np.exp(-(x**2 + y**2 + z**2) / 0.5**2), np.sin(np.pi * x) * y + z**3 - (x < 0)])
    np.testing.assert_allclose(got, want, rtol=1e-14, atol=1e-15)
    with pytest.raises(Exception):
        it.initialise_expressions(["exp(", "0"])


def tensor_desc(n, precision=TS_F64, dt=None):
    from treesap_b200 import TS_MODEL_TENSOR_WAVE

    n3 = (n, n, n) if np.isscalar(n) else tuple(n)
    return wave_desc(n3, 3, periodic=(1, 1, 1), ko=0.1, precision=precision, model=TS_MODEL_TENSOR_WAVE,
                     dt=dt if dt is not None else 0.25 / n3[0])


def test_tensor_model_matches_oracle(ctx, port_oracle):
    """12-component tensor wave (symmetric-tensor aliases, mixed derivatives, trace) vs the oracle."""
    d = tensor_desc((20, 17, 23))
    state = smooth_state(d.shape(), seed=33)
    it = Integrator(ctx, d)
    it.set_state(state)
    it.step(3)
    gpu = it.get_state()
    cpu, _, _ = port_oracle.run(d, 3, state=state)
    assert relerr(gpu, cpu) <= TOL_F64


def test_tensor_fp32_stage_error_vs_fp64(ctx):
    from treesap_b200 import TS_INIT_FOURIER

    rng = np.random.default_rng(3)
    modes = []
    for _ in range(12):
        k = rng.integers(-3, 4, 3)
        modes.append([rng.integers(0, 6), rng.normal(0, 0.01), *k, rng.uniform(0, 6.28)])
    out = {}
    for p in (TS_F64, TS_F32_STAGE):
        it = Integrator(ctx, tensor_desc(32, p))
        it.initialise(TS_INIT_FOURIER, np.array(modes, dtype=float))
        it.step(40)
        out[p] = it.get_state()
    ctx.sync()
    assert relerr(out[TS_F32_STAGE], out[TS_F64]) <= 1e-6


@pytest.mark.parametrize("n,ngrow,bcmode", [((4, 5, 4), 4, "periodic"), ((2, 6, 3), 2, "dirichlet"),
                                             ((1, 1, 7), 1, "periodic"), ((4, 4, 9), 4, "dirichlet"),
                                             ((3, 3, 3), 3, "periodic")])
def test_extents_at_the_ghost_width(ctx, port_oracle, n, ngrow, bcmode):
    """The smallest boxes the descriptor accepts (extents equal to the stencil half-width, so a
    periodic image spans the whole box; one-cell directions at ngrow 1), far smaller than one
    tile: RK4 FP64 against the oracle."""
    kw = dict(ko=0.1, dt=0.05)
    if bcmode == "periodic":
        d = wave_desc(n, ngrow, periodic=(1, 1, 1), **kw)
    else:
        d = wave_desc(n, ngrow, periodic=(0, 1, 0), bc=TS_BC_DIRICHLET, bc_values=(0.25, -0.5), **kw)
    state = smooth_state(d.shape(), seed=sum(n) + ngrow)
    it = Integrator(ctx, d)
    it.set_state(state)
    it.step(3)
    gpu = it.get_state()
    ctx.sync()
    cpu, _, _ = port_oracle.run(d, 3, state=state)
    assert np.isfinite(gpu).all()
    assert relerr(gpu, cpu) <= TOL_F64


def test_extents_below_the_ghost_width_are_rejected(ctx):
    from treesap_b200 import TSError

    with pytest.raises(TSError, match="INVALID_ARGUMENT"):
        Integrator(ctx, wave_desc((3, 8, 8), 4))


@pytest.mark.parametrize("precision", [TS_F64, TS_F32_STAGE])
def test_periodic_translation_equivariance_on_a_large_box(ctx, precision):
    """Size-independent property at 512 x 256 x 192 (16 x-tiles of 32 cells, several z chunks):
    on a periodic grid with uniform spacing the step commutes with a cyclic shift of the state,
    bit for bit, because every cell runs the same arithmetic on the same neighbour values."""
    n = (512, 256, 192)
    d = wave_desc(n, 4, periodic=(1, 1, 1), ko=0.2, precision=precision, prob_hi=(2.0, 1.0, 0.75), dt=0.25 / 256)
    rng = np.random.default_rng(3)
    state = np.zeros(d.shape())
    z, y, x = np.meshgrid(*(np.arange(m) / m for m in n[::-1]), indexing="ij")
    for c in range(2):
        for _ in range(3):
            k = rng.integers(-3, 4, 3)
            state[c] += rng.normal() * np.cos(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + rng.uniform(0, 6.28))
    shift = (5, -3, 7)  # cells along z, y, x
    outs = []
    for s in (state, np.roll(state, shift, axis=(1, 2, 3))):
        it = Integrator(ctx, d)
        it.set_state(s)
        it.step(2)
        outs.append(it.get_state())
        it.close()
    ctx.sync()
    assert np.abs(outs[0]).max() > 0.1
    assert np.array_equal(np.roll(outs[0], shift, axis=(1, 2, 3)), outs[1])
