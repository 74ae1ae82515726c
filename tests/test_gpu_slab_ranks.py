"""The multi-process slab integrator of the C ABI (ts_integrator_create_slab, ts_slab_*), as
one process runs it for several slabs on one GPU (treesap_b200.slabs.step_lockstep: the halo
exchange becomes device-to-device copies; across GPUs the same planes travel through NCCL,
treesap_b200.slabs.TorchComm). Each slab is initialised in global coordinates and the gathered
state after several steps must be bitwise the single box's (C2-like absorbing layer and
Dirichlet boundaries; periodic z, where the end slabs exchange with each other).
"""
import numpy as np
import pytest

import treesap_b200 as tsb
from treesap_b200.configs import c2_pulses, wave_desc
from treesap_b200.slabs import SlabDomain, step_lockstep

pytestmark = pytest.mark.gpu

CASES = {
    "c2-like": dict(n=(40, 36, 48), ngrow=4, periodic=(0, 0, 0), ko=0.2, abl_thickness=6, abl_max=10.0,
                    bc=tsb.TS_BC_DIRICHLET),
    "periodic": dict(n=(32, 28, 45), ngrow=2, periodic=(1, 1, 1), ko=0.1),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("world", [2, 3])
@pytest.mark.parametrize("scheme,precision", [(tsb.TS_RK4, tsb.TS_F64), (tsb.TS_EULER, tsb.TS_F64),
                                              (tsb.TS_RK4, tsb.TS_F32_STAGE)])
def test_rank_slabs_are_bitwise_the_single_box(ctx, case, world, scheme, precision):
    kw = dict(CASES[case])
    desc = wave_desc(kw.pop("n"), kw.pop("ngrow"), scheme=scheme, precision=precision, **kw)
    pulses = c2_pulses(5, 4)
    it = tsb.Integrator(ctx, desc)
    it.initialise(tsb.TS_INIT_GAUSSIAN, pulses)
    it.step(4)
    want = it.get_state()
    it.close()

    doms = [SlabDomain(desc, r, world, comm=None, ctx=ctx) for r in range(world)]
    for d in doms:
        d.slab.initialise(tsb.TS_INIT_GAUSSIAN, pulses)
    step_lockstep(doms, 4, stream=ctx.stream)
    got = np.concatenate([d.slab.get_state() for d in doms], axis=1)
    ctx.sync()
    for d in doms:
        d.slab.close()
    assert np.isfinite(want).all()
    assert np.array_equal(got, want)
