"""Host-side checks of the C++20 header front end (no GPU).

* Stencil weights / KO coefficients / tensor-alias maps printed by tests/cpp/probe_frontend.cpp
  against the exact rationals of the finite-difference formulas.
* The built-in models and the front end compile for sm_100a (nvcc cross-compile).
* Drop-in: the reference's own example right-hand sides (examples/01-wave-eqn/WaveEqnRHS.hpp,
  examples/02-temporaries/NonLinearRHS.hpp) compile UNCHANGED against these headers into the
  fused sm_100a stage kernels (skipped where the reference sources are absent).
"""
import json
import shutil
import subprocess
from fractions import Fraction
from math import comb, factorial
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
INC = ["-I", str(ROOT / "include"), "-I", str(ROOT / "treesap_b200/cpp/compat"), "-I",
       str(ROOT / "treesap_b200/cpp/treesap"), "-I", str(ROOT / "treesap_b200/cpp/rhs")]
from conftest import REFERENCE_SKIP, reference_root  # noqa: E402

REF = reference_root()


def first_w(n, p):
    if p == 0:
        return Fraction(0)
    return Fraction((-1) ** (p + 1) * factorial(n) ** 2, p * factorial(n - p) * factorial(n + p))


def second_w(n, p):
    if p == 0:
        return -2 * sum(Fraction(1, k * k) for k in range(1, n + 1))
    return Fraction(2 * (-1) ** (p + 1) * factorial(n) ** 2, p * p * factorial(n - p) * factorial(n + p))


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("probe") / "probe"
    subprocess.run(["g++", "-std=c++20", "-O1", *INC, str(ROOT / "tests/cpp/probe_frontend.cpp"), "-o", str(exe)],
                   check=True)
    return json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)


@pytest.mark.parametrize("n", [1, 2, 3, 4])
def test_weights_are_the_exact_rationals(probe, n):
    w = probe["weights"][str(n)]
    for p in range(n + 1):
        assert w["first"][p] == float(first_w(n, p))
        assert w["second"][p] == float(second_w(n, p))
        assert w["ko"][p] == -((-1) ** p) * comb(2 * n, n + p)


def test_weight_table_known_values(probe):
    # D1 / D2 weights of half-width 1..4 (standard centred finite-difference tables)
    d1 = {1: [1 / 2], 2: [2 / 3, -1 / 12], 3: [3 / 4, -3 / 20, 1 / 60], 4: [4 / 5, -1 / 5, 4 / 105, -1 / 280]}
    d2c = {1: -2.0, 2: -5 / 2, 3: -49 / 18, 4: -205 / 72}
    for n in (1, 2, 3, 4):
        w = probe["weights"][str(n)]
        assert w["first"][1:] == pytest.approx(d1[n], rel=1e-15)
        assert w["second"][0] == pytest.approx(d2c[n], rel=1e-15)


@pytest.mark.parametrize("n", [2, 3, 4])
def test_moment_conditions(probe, n):
    """D1 and D2 of half-width n are exact for polynomials of degree <= 2n."""
    w = probe["weights"][str(n)]
    for deg in range(2 * n + 1):
        m1 = sum(w["first"][p] * (p ** deg - (-p) ** deg) for p in range(1, n + 1))
        m2 = w["second"][0] * (1 if deg == 0 else 0) + sum(w["second"][p] * (p ** deg + (-p) ** deg)
                                                          for p in range(1, n + 1))
        assert m1 == pytest.approx(1.0 if deg == 1 else 0.0, abs=1e-12)
        assert m2 == pytest.approx(2.0 if deg == 2 else 0.0, abs=1e-12)


def test_tensor_alias_maps(probe):
    sym = {(a, b): c for a, b, c in probe["sym2"]}
    assert [sym[(0, 0)], sym[(1, 0)], sym[(1, 1)], sym[(2, 0)], sym[(2, 1)], sym[(2, 2)]] == [6, 7, 8, 9, 10, 11]
    assert all(sym[(a, b)] == sym[(b, a)] for a in range(3) for b in range(3))
    r2 = {(a, b): c for a, b, c in probe["rank2"]}
    assert all(r2[(a, b)] == 1 + a + 3 * b for a in range(3) for b in range(3))


def nvcc_compile(src: Path, out: Path, extra=()):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-std=c++20", "--expt-relaxed-constexpr", "--extended-lambda", "-gencode",
           "arch=compute_100a,code=sm_100a", *INC, *extra, "-c", str(src), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]


DROPIN = r'''
#include "integrators/SingleLevelEulerIntegrator.hpp"
#include "integrators/SingleLevelRK4Integrator.hpp"
#include "pde-model/PDEModel.hpp"
#include "pde-model/bcs/DirichletBC.hpp"
#include "init/ConstInit.hpp"
#include "%s"
using RHS = %s;
using Model = treesap::PDEModel<RHS, treesap::ConstInit<RHS::ncomp>, treesap::DirichletBC<RHS::ncomp, RHS::ngrow>>;
template class treesap::SingleLevelRK4Integrator<Model>;
template class treesap::SingleLevelEulerIntegrator<Model>;
'''


@pytest.mark.skipif(REF is None, reason=REFERENCE_SKIP)
@pytest.mark.parametrize("header,rhs", [("examples/01-wave-eqn/WaveEqnRHS.hpp", "WaveEqnRHS<2>"),
                                        ("examples/02-temporaries/NonLinearRHS.hpp", "NonLinearRHS<1>")])
def test_reference_example_rhs_compiles_unchanged(tmp_path, header, rhs):
    src = tmp_path / "dropin.cu"
    src.write_text(DROPIN % (str(REF / header), rhs))
    nvcc_compile(src, tmp_path / "dropin.o")


def test_bounds_checked_view_flags_out_of_range_reads(tmp_path):
    """TREESAP_B200_CHECK builds: the stencil view's range checks, run on the host (no GPU). An
    out-of-range read sets bit 2 (index out of bounds) of the error word and reads the centre;
    in-range reads are untouched. The GPU side of the same build is exercised by the
    bounds-checked tile variants (tests/test_gpu_tile_variants.py)."""
    exe = tmp_path / "check_view"
    subprocess.run(["g++", "-std=c++20", "-O1", *INC, str(ROOT / "tests/cpp/check_view_probe.cpp"), "-o", str(exe)],
                   check=True)
    r = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    assert r["in_plane"] == 34 and r["in_glob"] == 1000 + (8 * 35 + 4 * 5 + 3) and r["err_in"] == 0
    assert r["err_plane"] == 2 and r["out_plane"] == 17
    assert r["err_glob"] == 2 and r["out_glob"] == 1000 + 4 * 35 + 17


def test_quadratic_layer_sigma_matches_the_square_root_path(tmp_path):
    """The branch-free damping strength of a profile with of_square (QuadraticProfile) equals the
    reference's path (square root of the squared index distance, then the profile) to rounding
    at every cell of the layer, and is exactly 0 in the bulk."""
    exe = tmp_path / "abl_sigma"
    subprocess.run(["g++", "-std=c++20", "-O1", *INC, str(ROOT / "tests/cpp/abl_sigma_probe.cpp"), "-o", str(exe)],
                   check=True)
    r = json.loads(subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout)
    assert r["bulk_zero"] and r["layer_cells"] == 64**3 - 32**3
    assert r["worst_rel"] <= 4e-16
