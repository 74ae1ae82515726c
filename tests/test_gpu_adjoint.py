"""Discrete adjoint of RK4 for the variable-speed wave model (ts_adjoint_*).

Checks, on small periodic grids:
  * the adjoint's forward model is the library's KO + c(x)^2 wave model, bitwise;
  * the adjoint dot-product identity against the tangent-linear run:
      <dJ/du_T, du_T> = <g_phi0, dphi0> + <g_pi0, dpi0> + <g_c, dc>   (relative 1e-11);
  * gradients against central finite differences of the loss (relative 1e-5), for the
    initial state (J is quadratic in it) and for the speed c(x);
  * the result does not depend on the checkpoint interval (bitwise).
"""
import numpy as np
import pytest

from treesap_b200 import Adjoint, Integrator, TSError
from treesap_b200.configs import c5_pulse, c5_speed, wave_desc

pytestmark = pytest.mark.gpu


def setup(n=24, ngrow=2, ko=0.1, seed=1):
    d = wave_desc(n, ngrow, periodic=(1, 1, 1), ko=ko)
    c = c5_speed(n, seed=seed, modes=6, kmax=3)
    phi0 = c5_pulse(n, width=0.15)
    pi0 = 0.1 * c5_pulse(n, shift_cells=3, width=0.2)
    target = c5_pulse(n, shift_cells=2, amplitude=1.05, width=0.15)
    return d, c, phi0, pi0, target


@pytest.mark.parametrize("ngrow", [2, 4])
def test_adjoint_forward_is_the_library_model(ctx, ngrow):
    d, c, phi0, pi0, _ = setup(20, ngrow)
    adj = Adjoint(ctx, d, 5)
    phi, pi = adj.forward(phi0, pi0, c, 12)
    it = Integrator(ctx, d, c2=c * c)
    it.set_state(np.stack([phi0, pi0]))
    it.step(12)
    ref = it.get_state()
    assert np.array_equal(phi, ref[0]) and np.array_equal(pi, ref[1])


@pytest.mark.parametrize("ngrow", [2, 4])
def test_adjoint_dot_product_identity(ctx, ngrow):
    d, c, phi0, pi0, target = setup(24, ngrow)
    nsteps = 15
    adj = Adjoint(ctx, d, 4)
    rng = np.random.default_rng(7)
    dphi0, dpi0, dc = (rng.standard_normal(phi0.shape) for _ in range(3))
    loss, gphi, gpi, gc = adj.gradient(phi0, pi0, c, nsteps, target)
    phiT, _ = adj.forward(phi0, pi0, c, nsteps)
    dphiT, _ = adj.tangent(phi0, pi0, c, dphi0, dpi0, dc, nsteps)
    lhs = float(np.sum((phiT - target) * dphiT))
    rhs = float(np.sum(gphi * dphi0) + np.sum(gpi * dpi0) + np.sum(gc * dc))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs)), (lhs, rhs)
    assert loss == pytest.approx(0.5 * float(np.sum((phiT - target) ** 2)), rel=1e-14)


def test_adjoint_gradient_matches_central_differences(ctx):
    d, c, phi0, pi0, target = setup(24, 2)
    nsteps = 20
    adj = Adjoint(ctx, d, 6)
    _, gphi, gpi, gc = adj.gradient(phi0, pi0, c, nsteps, target)
    rng = np.random.default_rng(11)

    def loss(p0, c_):
        phiT, _ = adj.forward(p0, pi0, c_, nsteps)
        return 0.5 * float(np.sum((phiT - target) ** 2))

    for _ in range(3):
        v = rng.standard_normal(phi0.shape)
        v /= np.linalg.norm(v)
        eps = 1e-3
        fd = (loss(phi0 + eps * v, c) - loss(phi0 - eps * v, c)) / (2 * eps)
        ad = float(np.sum(gphi * v))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)
    for _ in range(3):
        v = rng.standard_normal(c.shape)
        v /= np.linalg.norm(v)
        eps = 1e-5
        fd = (loss(phi0, c + eps * v) - loss(phi0, c - eps * v)) / (2 * eps)
        ad = float(np.sum(gc * v))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def test_adjoint_checkpoint_interval_does_not_change_the_result(ctx):
    d, c, phi0, pi0, target = setup(16, 2)
    out = []
    for every in (1, 7, 30):
        adj = Adjoint(ctx, d, every)
        out.append(adj.gradient(phi0, pi0, c, 13, target))
    for o in out[1:]:
        assert o[0] == out[0][0]
        for a, b in zip(o[1:], out[0][1:]):
            assert np.array_equal(a, b)


def test_adjoint_rejects_unsupported(ctx):
    with pytest.raises(TSError) as e:
        Adjoint(ctx, wave_desc(16, 2, periodic=(1, 1, 0), ko=0.1))
    assert e.value.status == 2
    with pytest.raises(TSError) as e:
        Adjoint(ctx, wave_desc(16, 3, periodic=(1, 1, 1)))
    assert e.value.status == 2


def relmax(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("ngrow", [2, 4])
def test_fp32_stage_state_gradient_vs_fp64(ctx, ngrow):
    """FP32-stage forward run and reverse sweep: loss and initial-state gradients within 1e-6 of FP64."""
    d, c, phi0, pi0, target = setup(24, ngrow)
    adj = Adjoint(ctx, d, 5)
    l64, g64, p64, _ = adj.gradient(phi0, pi0, c, 20, target)
    l32, g32, p32, c32 = adj.gradient_f32(phi0, pi0, c, 20, target, speed=False)
    assert c32 is None
    assert abs(l32 - l64) <= 1e-6 * abs(l64)
    assert relmax(g32, g64) <= 1e-6 and relmax(p32, p64) <= 1e-6


@pytest.mark.parametrize("ngrow,every,nsteps", [(2, 5, 20), (4, 7, 17), (2, 30, 13), (2, 1, 6)])
def test_fp32_stage_speed_gradient_vs_fp64(ctx, ngrow, every, nsteps):
    """FP32-stage speed gradient (forward and adjoint registers of each step recomputed from
    checkpoints) within 1e-6 of the FP64 speed gradient, for checkpoint intervals that divide
    the run, that do not, that exceed it and of one step; the state gradient is the one of the
    state-only call, bitwise."""
    d, c, phi0, pi0, target = setup(24, ngrow)
    adj = Adjoint(ctx, d, every)
    l64, g64, p64, c64 = adj.gradient(phi0, pi0, c, nsteps, target)
    l32, g32, p32, c32 = adj.gradient_f32(phi0, pi0, c, nsteps, target)
    _, g32s, p32s, _ = adj.gradient_f32(phi0, pi0, c, nsteps, target, speed=False)
    assert abs(l32 - l64) <= 1e-6 * abs(l64)
    assert relmax(c32, c64) <= 1e-6, relmax(c32, c64)
    assert np.array_equal(g32, g32s) and np.array_equal(p32, p32s)


def test_fp32_stage_state_gradient_matches_central_differences(ctx):
    d, c, phi0, pi0, target = setup(20, 2)
    adj = Adjoint(ctx, d, 5)
    _, g32, _, _ = adj.gradient_f32(phi0, pi0, c, 12, target, speed=False)
    rng = np.random.default_rng(5)
    for _ in range(3):
        v = rng.standard_normal(phi0.shape)
        v /= np.linalg.norm(v)
        # J is quadratic in the initial state, so the central difference carries no truncation
        # error at any step; a wide step keeps the FP32-stage rounding of J (about 1e-8 of J)
        # small against the difference itself.
        eps = 0.1
        lp = adj.gradient_f32(phi0 + eps * v, pi0, c, 12, target, speed=False)[0]
        lm = adj.gradient_f32(phi0 - eps * v, pi0, c, 12, target, speed=False)[0]
        fd = (lp - lm) / (2 * eps)
        ad = float(np.sum(g32 * v))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def test_fp32_stage_speed_gradient_matches_central_differences(ctx):
    """<dJ/dc, v> of the FP32-stage form against central differences of the FP64 loss (the
    FP32-stage loss rounds at about 1e-8 of J, too coarse for a difference quotient in c)."""
    d, c, phi0, pi0, target = setup(24, 2)
    nsteps = 20
    adj = Adjoint(ctx, d, 6)
    _, _, _, gc = adj.gradient_f32(phi0, pi0, c, nsteps, target)
    rng = np.random.default_rng(12)

    def loss(c_):
        phiT, _ = adj.forward(phi0, pi0, c_, nsteps)
        return 0.5 * float(np.sum((phiT - target) ** 2))

    for _ in range(3):
        v = rng.standard_normal(c.shape)
        v /= np.linalg.norm(v)
        eps = 1e-5
        fd = (loss(c + eps * v) - loss(c - eps * v)) / (2 * eps)
        ad = float(np.sum(gc * v))
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)
