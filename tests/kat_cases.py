"""Analytic known-answer cases (from the mathematics of the scheme, not from any implementation).

* polynomial exactness: centred D2 of half-width g is exact for polynomials of degree <= 2g,
  and Kreiss-Oliger of order r annihilates polynomials of degree < 2r;
* single periodic Fourier mode: the discrete operator acts on cos(2 pi k.x) by its symbol,
  so one RK4 step multiplies (phi_hat, pi_hat) by R(dt A) = I + Z + Z^2/2 + Z^3/6 + Z^4/24.
"""
from fractions import Fraction
from math import comb, factorial

import numpy as np


def d2_weights(n):
    w = [-2 * sum(Fraction(1, k * k) for k in range(1, n + 1))]
    w += [Fraction(2 * (-1) ** (p + 1) * factorial(n) ** 2, p * p * factorial(n - p) * factorial(n + p))
          for p in range(1, n + 1)]
    return [float(x) for x in w]


def d2_symbol(n, theta, dx):
    """Eigenvalue of the centred D2 on exp(i theta j): (w0 + 2 sum_s w_s cos(s theta)) / dx^2."""
    w = d2_weights(n)
    return (w[0] + 2 * sum(w[s] * np.cos(s * theta) for s in range(1, n + 1))) / dx**2


def ko_symbol(r, theta, dx):
    """Eigenvalue of D_KO = -(1/dx) 2^{-2r} sum_m (-1)^m C(2r, r+m) f_m on exp(i theta j)."""
    s = comb(2 * r, r) + 2 * sum((-1) ** m * comb(2 * r, r + m) * np.cos(m * theta) for m in range(1, r + 1))
    return -s / (2 ** (2 * r) * dx)


def fourier_case(n, ngrow, kvec, ko, dt):
    """Returns (state0, exact state after one RK4 step) for phi0 = cos(2 pi k.x), pi0 = 0, on [0,1)^3."""
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) * dx
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    arg = 2 * np.pi * (kvec[0] * X + kvec[1] * Y + kvec[2] * Z)
    lam = sum(d2_symbol(ngrow, 2 * np.pi * k * dx, dx) for k in kvec)
    kap = ko * sum(ko_symbol(ngrow, 2 * np.pi * k * dx, dx) for k in kvec)
    A = np.array([[kap, 1.0], [lam, kap]])
    Zm = dt * A
    R = np.eye(2) + Zm + Zm @ Zm / 2 + Zm @ Zm @ Zm / 6 + Zm @ Zm @ Zm @ Zm / 24
    s0 = np.stack([np.cos(arg), np.zeros_like(arg)])
    s1 = np.stack([R[0, 0] * np.cos(arg), R[1, 0] * np.cos(arg)])
    return s0, s1


def polynomial_case(n, ngrow):
    """phi0 = polynomial of degree 2 ngrow on [0,1]^3, pi0 = 0; returns (state0, Laplacian, interior mask)."""
    dx = 1.0 / n
    x = (np.arange(n) + 0.5) * dx
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    p = 2 * ngrow
    phi = X**p + 0.5 * Y ** (p - 1) * Z + 0.25 * Z**p + X * Y
    lap = p * (p - 1) * X ** (p - 2) + 0.5 * (p - 1) * (p - 2) * Y ** (p - 3) * Z + 0.25 * p * (p - 1) * Z ** (p - 2)
    interior = np.zeros_like(phi, dtype=bool)
    interior[ngrow:n - ngrow, ngrow:n - ngrow, ngrow:n - ngrow] = True
    return np.stack([phi, np.zeros_like(phi)]), lap, interior
