"""Analytic known-answer tests of the oracle (CPU); the GPU path runs the same cases in
tests/test_gpu_kat.py."""
import numpy as np
import pytest

from kat_cases import fourier_case, polynomial_case
from treesap_b200 import TS_EULER
from treesap_b200.configs import wave_desc


@pytest.mark.parametrize("ngrow", [1, 2, 3, 4])
@pytest.mark.parametrize("ko", [0.0, 0.2])
def test_fourier_mode_one_rk4_step(port_oracle, ngrow, ko):
    n, dt = 16, 0.2 / 16
    s0, s1 = fourier_case(n, ngrow, (2, 1, 3), ko, dt)
    got, _, _ = port_oracle.run(wave_desc(n, ngrow, ko=ko, dt=dt), 1, state=s0)
    assert np.abs(got - s1).max() <= 1e-12 * np.abs(s1).max() * 100


@pytest.mark.parametrize("ngrow", [1, 2, 3, 4])
def test_polynomial_exactness_euler(port_oracle, ngrow):
    n, dt = 14, 1e-3
    s0, lap, interior = polynomial_case(n, ngrow)
    got, _, _ = port_oracle.run(wave_desc(n, ngrow, periodic=(0, 0, 0), dt=dt, scheme=TS_EULER), 1, state=s0)
    rhs_pi = got[1] / dt
    assert np.abs(rhs_pi - lap)[interior].max() <= 1e-6 * np.abs(lap).max()
    assert np.array_equal(got[0], s0[0])  # phi_t = pi0 = 0


@pytest.mark.parametrize("r", [1, 2, 3, 4])
def test_ko_annihilates_low_degree(port_oracle, r):
    """KO of order r annihilates polynomials of degree < 2r: phi stays put under Euler with pi0 = 0."""
    n, dt = 14, 1e-3
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) * dx
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    phi = X ** (2 * r - 1) + Y * Z
    s0 = np.stack([phi, np.zeros_like(phi)])
    got, _, _ = port_oracle.run(wave_desc(n, r, periodic=(0, 0, 0), ko=0.3, dt=dt, scheme=TS_EULER), 1, state=s0)
    interior = np.zeros_like(phi, dtype=bool)
    interior[r:n - r, r:n - r, r:n - r] = True
    assert np.abs(got[0] - phi)[interior].max() <= 1e-9
