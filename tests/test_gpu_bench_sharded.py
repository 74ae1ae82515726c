"""The multi-GPU branch of bench.py (run_sharded: one 256 x 256 x 256N domain in N z slabs, a
halo exchange every RK4 stage) driven with a single rank on one GPU.

With one rank the slab covers the whole domain and there is no neighbour, so nothing is
exchanged and no collective runs; everything else of the branch runs as it does on N GPUs:
the slab integrator of the C ABI (ts_integrator_create_slab, ts_slab_*), SlabDomain's stage
loop, the stream-ordered timing, the end-to-end leg and the JSON line. The slab result must
equal the whole-box integrator's, bitwise (the same kernels on the same cells).
"""
import argparse
import contextlib
import io
import json

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sharded_branch_with_one_rank_prints_a_valid_line():
    import bench

    out = io.StringIO()
    with contextlib.redirect_stdout(out):
        bench.run_sharded(argparse.Namespace(steps=2, warmup=1), 0, 1, 0)
    line = json.loads(out.getvalue().strip().splitlines()[-1])
    assert line["n_gpus"] == 1 and line["steps"] == 2 and line["scaling"] == "weak"
    assert line["value"] > 0 and line["fp64"]["value"] > 0
    assert line["config"]["grid"] == [256, 256, 256]
    assert line["gpu_launches"] == 2 * 4  # one stage kernel per stage, no neighbour to exchange with
    assert line["e2e"]["value"] > 0 and line["e2e"]["h2d_bytes_per_step"] > 0


def test_single_rank_slab_matches_the_whole_box():
    import treesap_b200 as tsb
    from treesap_b200.configs import c2_pulses, wave_desc
    from treesap_b200.slabs import SlabDomain, TorchComm

    ctx = tsb.Context(0)
    d = wave_desc((40, 36, 48), 4, periodic=(0, 0, 0), ko=0.2, abl_thickness=6, abl_max=10.0,
                  bc=tsb.TS_BC_DIRICHLET, precision=tsb.TS_F32_STAGE)
    pulses = c2_pulses(4, 3)
    whole = tsb.Integrator(ctx, d)
    whole.initialise(tsb.TS_INIT_GAUSSIAN, pulses)
    whole.step(3)
    want = whole.get_state()
    dom = SlabDomain(d, 0, 1, TorchComm(ctx.stream), ctx=ctx)
    dom.slab.initialise(tsb.TS_INIT_GAUSSIAN, pulses)
    dom.step(3)
    got = dom.slab.get_state()
    assert np.array_equal(got, want)
    dom.slab.close()
    whole.close()
    ctx.close()
