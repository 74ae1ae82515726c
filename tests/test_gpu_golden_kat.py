"""The B200 path (through the C ABI) against the reference's golden fixtures and the analytic
known-answer cases. FP64 plain form: relative max-norm <= 1e-12."""
import numpy as np
import pytest

from golden_cases import load, names
from kat_cases import fourier_case, polynomial_case
from treesap_b200 import TS_BC_DIRICHLET, TS_BC_NOOP, TS_EULER, TS_INIT_GAUSSIAN, TS_RK4, Integrator, WaveDesc
from treesap_b200.configs import wave_desc

pytestmark = pytest.mark.gpu
TOL = 1e-12


def wave_desc_from_golden(d) -> WaveDesc:
    w = WaveDesc()
    w.n[:] = [int(v) for v in d["n"]]
    w.prob_lo[:] = [float(v) for v in d["prob_lo"]]
    w.prob_hi[:] = [float(v) for v in d["prob_hi"]]
    w.periodic[:] = [int(v) for v in d["periodic"]]
    w.ngrow = int(d["ngrow"])
    w.model = int(d["model"])
    w.ko_strength = float(d["ko_strength"])
    w.abl_thickness = int(d["abl_thickness"])
    w.abl_max_strength = float(d["abl_max_strength"])
    w.abl_profile = int(d["abl_profile"])
    w.bc = int(d["bc"])
    w.bc_values[:] = [float(v) for v in d["bc_values"]]
    w.dt = float(d["dt"])
    w.scheme = int(d["integrator"])
    w.precision = 0
    return w


# the library builds the tensor model for ngrow 3 only (its benchmark configuration)
@pytest.mark.parametrize("name", [n for n in names() if not n.startswith("tensor") or n.endswith("_g3")])
def test_gpu_reproduces_reference_golden(ctx, name):
    d, inp, nsteps, t, out = load(name)
    w = wave_desc_from_golden(d)
    it = Integrator(ctx, w, c2=inp.get("c2"))
    if "state" in inp:
        it.set_state(inp["state"])
    else:
        it.initialise(int(inp.get("kind", TS_INIT_GAUSSIAN)), inp["items"])
    it.step(nsteps)
    got = it.get_state()
    ctx.sync()
    assert float(np.abs(got - out).max() / np.abs(out).max()) <= TOL
    tt, s = it.time()
    assert s == nsteps and abs(tt - t) <= 1e-15


@pytest.mark.parametrize("ngrow", [1, 2, 3, 4])
@pytest.mark.parametrize("ko", [0.0, 0.2])
def test_gpu_fourier_mode_one_rk4_step(ctx, ngrow, ko):
    n, dt = 16, 0.2 / 16
    s0, s1 = fourier_case(n, ngrow, (2, 1, 3), ko, dt)
    it = Integrator(ctx, wave_desc(n, ngrow, ko=ko, dt=dt))
    it.set_state(s0)
    it.step(1)
    got = it.get_state()
    assert np.abs(got - s1).max() <= 1e-10 * np.abs(s1).max()


@pytest.mark.parametrize("ngrow", [1, 2, 3, 4])
def test_gpu_polynomial_exactness(ctx, ngrow):
    n, dt = 14, 1e-3
    s0, lap, interior = polynomial_case(n, ngrow)
    it = Integrator(ctx, wave_desc(n, ngrow, periodic=(0, 0, 0), dt=dt, scheme=TS_EULER))
    it.set_state(s0)
    it.step(1)
    got = it.get_state()
    assert np.abs(got[1] / dt - lap)[interior].max() <= 1e-6 * np.abs(lap).max()


@pytest.mark.parametrize("n", [(4, 4, 4), (5, 7, 4), (64, 3, 9), (300, 12, 5)])
def test_gpu_edge_sizes(ctx, port_oracle, n):
    """Domains narrower than a tile, equal to the ghost width, and wider than several tiles."""
    g = min(4, min(n))
    d = wave_desc(n, g, periodic=(1, 0, 1), ko=0.1, bc=TS_BC_DIRICHLET, bc_values=(0.2, 0.0), dt=0.1 / max(n))
    rng = np.random.default_rng(sum(n))
    s = rng.standard_normal(d.shape())
    it = Integrator(ctx, d)
    it.set_state(s)
    it.step(3)
    got = it.get_state()
    cpu, _, _ = port_oracle.run(d, 3, state=s)
    assert float(np.abs(got - cpu).max() / np.abs(cpu).max()) <= TOL


def test_gpu_invalid_descriptor_is_rejected(ctx):
    from treesap_b200 import TSError

    d = wave_desc(16, 5)  # ngrow 5 is outside 1..4
    with pytest.raises(TSError):
        Integrator(ctx, d)
    d = wave_desc(16, 2, scheme=TS_EULER, precision=1)  # FP32-stage needs RK4
    with pytest.raises(TSError):
        Integrator(ctx, d)
