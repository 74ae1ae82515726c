"""The reference's own example models, compiled unchanged, on the B200 against the reference.

examples/01-wave-eqn/WaveEqnRHS.hpp (the first-order wave system phi_t = div u, u_t = grad phi:
four components, first-derivative stencils) and examples/02-temporaries/NonLinearRHS.hpp (a
nonlinear wave equation whose RHS keeps pi in a Workspace Temporary loaded by component 0 and
reused by component 1) are compiled unchanged twice by the oracle recipe: against the B200
front end into the fused sm_100a stage kernels (oracle/_ref/libtsb_examples.so) and against
the reference's own headers and integrators on the host (oracle/_ref/libtsref_examples.so).
Both sides step the same seeded state; the GPU result must match the reference to 1e-12
relative max-norm (the plain form's bar) for every ngrow 1..4, with and without Kreiss-Oliger,
Dirichlet and periodic boundaries, RK4 and Euler, one box and several (block_size).

The same holds for DerivativeProbeRHS (tests/cpp), a test-only model that runs the first- and
third-derivative stencils, unmixed and mixed, that the built-in models never use. Being linear,
the probe also runs in the FP32-stage RK4 form, checked against the reference's FP64 RK4 at
1e-6.
"""
import numpy as np
import pytest

from oracle import pyoracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (pyoracle.examples_available("ref") and pyoracle.examples_available("gpu")),
                                 reason="example-model libraries not built (oracle recipe with the reference sources)")]
TOL = 1e-12


def desc(n, ngrow, *, periodic=(0, 0, 0), ko=0.0, bc=1, bc_values=(0.0,) * 4, integrator=1, block=(0, 0, 0),
         cfl=0.2):
    d = pyoracle.RefDesc()
    d.n[:] = list(n)
    d.prob_lo[:] = [-1.0, -1.0, -1.0]
    d.prob_hi[:] = [-1.0 + 2.0 * n[0] / n[0], -1.0 + 2.0 * n[1] / n[0], -1.0 + 2.0 * n[2] / n[0]]
    d.periodic[:] = list(periodic)
    d.ngrow = ngrow
    d.model = 0
    d.ko_strength = ko
    d.abl_thickness = 0
    d.bc = bc
    for q, v in enumerate(bc_values):
        d.bc_values[q] = v
    d.dt = cfl * 2.0 / n[0]
    d.integrator = integrator
    d.block[:] = list(block)
    return d


def initial_state(example, n, seed):
    rng = np.random.default_rng(seed)
    nc = pyoracle.EXAMPLE_NCOMP[example]
    z, y, x = np.meshgrid(*(np.linspace(-1, 1, m, endpoint=False) + 1.0 / m for m in (n[2], n[1], n[0])),
                          indexing="ij")
    out = np.empty((nc, n[2], n[1], n[0]))
    for c in range(nc):
        cx, cy, cz = rng.uniform(-0.3, 0.3, 3)
        w = rng.uniform(0.3, 0.5)
        out[c] = rng.uniform(0.5, 1.0) * np.exp(-((x - cx) ** 2 + (y - cy) ** 2 + (z - cz) ** 2) / w**2)
    return out


@pytest.fixture(scope="module")
def sides():
    return pyoracle.ExampleRunner("ref"), pyoracle.ExampleRunner("gpu")


def relerr(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


CASES = []
for ex in (1, 2, 3):
    for g in (1, 2, 3, 4):
        if ex == 3 and g < 2:
            continue
        CASES.append((ex, g, (0, 0, 0), 0.0, 1, 1, (0, 0, 0)))
    CASES.append((ex, 2, (1, 1, 1), 0.1, 0, 1, (0, 0, 0)))  # periodic, Kreiss-Oliger
    CASES.append((ex, 3, (0, 1, 0), 0.0, 1, 0, (0, 0, 0)))  # mixed boundaries, Euler
    CASES.append((ex, 2, (0, 0, 0), 0.05, 1, 1, (16, 12, 8)))  # several boxes (block_size)


@pytest.mark.parametrize("example,ngrow,periodic,ko,bc,integrator,block", CASES)
def test_example_model_matches_reference(sides, example, ngrow, periodic, ko, bc, integrator, block):
    ref, gpu = sides
    n = (29, 23, 19)
    d = desc(n, ngrow, periodic=periodic, ko=ko, bc=bc, bc_values=(0.05, 0.0, 0.0, 0.0), integrator=integrator,
             block=block)
    s0 = initial_state(example, n, seed=100 * example + ngrow)
    gamma = 0.3 if example == 2 else 0.0
    want = ref.run(example, d, s0, 6, gamma)
    got = gpu.run(example, d, s0, 6, gamma)
    assert np.isfinite(got).all()
    assert relerr(got, want) <= TOL
    assert relerr(want, s0) > 1e-6  # the model moved the state


def test_nonlinear_example_is_nonlinear(sides):
    """NonLinearRHS's gamma term changes the result (the Workspace temporary is used)."""
    _, gpu = sides
    n = (24, 20, 16)
    d = desc(n, 2)
    s0 = initial_state(2, n, seed=9)
    a = gpu.run(2, d, s0, 4, 0.0)
    b = gpu.run(2, d, s0, 4, 0.5)
    assert relerr(a, b) > 1e-8


@pytest.mark.parametrize("ngrow,periodic,ko", [(2, (0, 0, 0), 0.0), (3, (1, 1, 1), 0.1), (4, (0, 1, 0), 0.05)])
def test_derivative_probe_in_the_fp32_stage_form(sides, ngrow, periodic, ko):
    """The D1/D3 probe (linear, value-type generic) in the FP32-stage RK4 form: its FP32
    stencils of the stage differences stay within 1e-6 of the reference's FP64 RK4."""
    ref, gpu = sides
    n = (29, 23, 19)
    d = desc(n, ngrow, periodic=periodic, ko=ko, bc=1, bc_values=(0.05, 0.0), integrator=1)
    s0 = initial_state(3, n, seed=300 + ngrow)
    want = ref.run(3, d, s0, 6, 0.0)
    d.integrator = 2  # the front end's FP32-stage RK4
    got = gpu.run(3, d, s0, 6, 0.0)
    assert np.isfinite(got).all()
    err = relerr(got, want)
    assert err <= 1e-6, err
    assert err > 0.0  # the FP32 stages did run (FP64 would agree to ~1e-15)
