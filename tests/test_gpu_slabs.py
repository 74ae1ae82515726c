"""block_size as z slabs (ts_wave_desc.block, integrators/ZSlabDomain.hpp).

The reference decomposes its domain into boxes of at most block_size cells
(SingleLevelIntegrator.hpp:47-49, 172-176) whose ghost cells FillPatch fills from the
neighbouring boxes (:153-163); the result does not depend on the decomposition. Here
block[2] < n[2] cuts the domain into z slabs whose ghost planes are exchanged every stage.
Checks: every slab decomposition gives bitwise the single box's state (absorbing layer,
Kreiss-Oliger, Dirichlet, periodic and mixed boundaries, RK4 and Euler, uneven slabs), and
matches the CPU oracle run with the same block_size (<= 1e-12); the FP32-stage form is bitwise
its single box too. Slabs thinner than the ghost width are refused.
"""
import numpy as np
import pytest

import treesap_b200 as tsb
from treesap_b200.configs import c2_pulses, wave_desc

pytestmark = pytest.mark.gpu

CASES = {
    "c2-like": dict(n=(40, 36, 60), ngrow=4, periodic=(0, 0, 0), ko=0.2, abl_thickness=6, abl_max=10.0,
                    bc=tsb.TS_BC_DIRICHLET),
    "periodic": dict(n=(32, 28, 45), ngrow=2, periodic=(1, 1, 1), ko=0.1),
    "periodic z only": dict(n=(30, 26, 33), ngrow=3, periodic=(0, 0, 1), ko=0.05, bc=tsb.TS_BC_DIRICHLET,
                            bc_values=(0.1, -0.2)),
    "x-y periodic, Dirichlet z": dict(n=(24, 24, 40), ngrow=1, periodic=(1, 1, 0), bc=tsb.TS_BC_DIRICHLET,
                                      bc_values=(0.3, 0.0)),
}


def make(case, block_z=0, scheme=tsb.TS_RK4, precision=tsb.TS_F64):
    kw = dict(CASES[case])
    n = kw.pop("n")
    return wave_desc(n, kw.pop("ngrow"), scheme=scheme, precision=precision, block=(0, 0, block_z), **kw)


def run(ctx, desc, steps, state=None):
    it = tsb.Integrator(ctx, desc)
    if state is None:
        it.initialise(tsb.TS_INIT_GAUSSIAN, c2_pulses(5, 4))
    else:
        it.set_state(state)
    it.step(steps)
    out = it.get_state()
    ctx.sync()
    it.close()
    return out


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("scheme,precision", [(tsb.TS_RK4, tsb.TS_F64), (tsb.TS_EULER, tsb.TS_F64),
                                              (tsb.TS_RK4, tsb.TS_F32_STAGE)])
@pytest.mark.parametrize("slabs", [2, 3, 5])
def test_slabs_are_bitwise_the_single_box(ctx, case, scheme, precision, slabs):
    whole = make(case, scheme=scheme, precision=precision)
    nz, g = whole.n[2], whole.ngrow
    block = -(-nz // slabs)  # ceil: `slabs` slabs of near-equal depth
    if nz // slabs < g:
        pytest.skip("slabs thinner than the ghost width")
    want = run(ctx, whole, 5)
    got = run(ctx, make(case, block, scheme=scheme, precision=precision), 5)
    assert np.isfinite(want).all()
    assert np.array_equal(got, want)


@pytest.mark.parametrize("case", ["c2-like", "periodic z only"])
def test_slabs_match_oracle_with_the_same_block_size(ctx, oracle, case):
    d = make(case, 13)
    rng = np.random.default_rng(21)
    s0 = rng.standard_normal(d.shape()) * 0.1
    got = run(ctx, d, 4, state=s0)
    want, _, _ = oracle.run(d, 4, state=s0, block=(d.n[0], d.n[1], 13))
    assert float(np.abs(got - want).max() / np.abs(want).max()) <= 1e-12


def test_slab_state_round_trip_and_time(ctx):
    d = make("periodic", 9)
    rng = np.random.default_rng(5)
    s = rng.standard_normal(d.shape())
    it = tsb.Integrator(ctx, d)
    it.set_state(s)
    assert np.array_equal(it.get_state(), s)
    it.step(3)
    t, n = it.time()
    assert n == 3 and abs(t - 3 * d.dt) < 1e-15
    it.close()


def test_thin_slabs_are_refused(ctx):
    with pytest.raises(tsb.TSError) as e:
        tsb.Integrator(ctx, make("c2-like", 3))  # 3 planes < ngrow 4
    assert e.value.status == 1
