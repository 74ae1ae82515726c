"""Parity at the benchmarked sizes: the GPU FP64 form against the CPU checker (the reference
build where present, else the plain-C restatement) on the benchmark configurations themselves,
so that size-dependent code (z chunking, tile heights, multi-wave grids, absorbing layers thicker
than a tile, the batched work list of uneven boxes) meets the oracle:

  C2  256^3, 8th order, KO 0.2, absorbing layer 16 cells (s^2, max 10), Dirichlet 0, 3 steps
  C3  192^3 tensorial wave (12 components, ngrow 3, KO 0.1), 32 Fourier modes, 2 steps
  C4  all 512 periodic instances (edges 16..96, ngrow 2) in one batch, 2 steps
  C5  the variable-speed forward model at 128^3 (ngrow 2, KO 0.1, seeded c(x)), 5 steps

Bar: relative max-norm <= 1e-12 (the plain form's tolerance).
"""
import numpy as np
import pytest

import treesap_b200 as tsb
from treesap_b200.configs import (c2_desc, c2_pulses, c3_desc, c3_modes, c4_descs, c4_pulses, c5_desc, c5_pulse,
                                  c5_speed)

pytestmark = pytest.mark.gpu
TOL = 1e-12


def relerr(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def test_c2_256_fp64_matches_oracle(ctx, oracle):
    d = c2_desc(tsb.TS_F64, 256)
    pulses = c2_pulses()
    it = tsb.Integrator(ctx, d)
    it.initialise(tsb.TS_INIT_GAUSSIAN, pulses)
    it.step(3)
    got = it.get_state()
    it.close()
    want, _, _ = oracle.run(d, 3, items=pulses)
    assert relerr(got, want) <= TOL


def test_c3_192_fp64_matches_oracle(ctx, oracle):
    d = c3_desc(tsb.TS_F64, 192)
    modes = c3_modes()
    it = tsb.Integrator(ctx, d)
    it.initialise(tsb.TS_INIT_FOURIER, modes)
    it.step(2)
    got = it.get_state()
    it.close()
    want, _, _ = oracle.run(d, 2, init_kind=2, items=modes)
    assert relerr(got, want) <= TOL


def test_c4_all_instances_fp64_match_oracle(ctx, oracle):
    descs = c4_descs(tsb.TS_F64)
    pulses = c4_pulses()
    b = tsb.Batch(ctx, descs)
    for i, p in enumerate(pulses):
        b.initialise(i, tsb.TS_INIT_GAUSSIAN, p)
    b.step(2)
    ctx.sync()
    worst = 0.0
    for i, (d, p) in enumerate(zip(descs, pulses)):
        want, _, _ = oracle.run(d, 2, items=p)
        worst = max(worst, relerr(b.get_state(i), want))
    b.close()
    assert worst <= TOL


def test_c5_forward_128_matches_oracle(ctx, oracle):
    d = c5_desc(128)
    c = c5_speed(128)
    c2 = c * c
    s0 = np.stack([c5_pulse(128), np.zeros((128, 128, 128))])
    it = tsb.Integrator(ctx, d, c2=c2)
    it.set_state(s0)
    it.step(5)
    got = it.get_state()
    it.close()
    want, _, _ = oracle.run(d, 5, state=s0, c2=c2)
    assert relerr(got, want) <= TOL
