"""Workload descriptors of the benchmark configurations (seeded synthetic inputs).

  C1  64^3 unit cube, periodic, scalar wave, 4th-order stencils (ngrow 2), KO 0.1, RK4,
      dt = 0.25 dx, 100 steps; phi0 = exp(-|x - c|^2 / 0.1^2), c = (1/2, 1/2, 1/2), pi0 = 0.
  C2  256^3 unit cube, scalar wave, 8th-order (ngrow 4), KO 0.2, absorbing layer 16 cells,
      profile s^2, max strength 10/L, targets 0 (Dirichlet-0 ghosts), RK4 dt = 0.25 dx,
      1000 steps; phi0 = sum of 8 Gaussians, A ~ U[0.5, 1], w ~ U[0.05, 0.15],
      c ~ U[0.25, 0.75]^3, pi0 = 0; FP64 and FP32-stage.
  C4  512 independent instances, cube edges n ~ U{16, 24, ..., 96}, unit cube (dx = 1/n),
      periodic, 4th-order stencils (ngrow 2), no KO, RK4 dt = 0.25/n each, 200 steps;
      one Gaussian per instance, A ~ U[0.5, 1], w ~ U[0.05, 0.2], c ~ U[0.3, 0.7]^3;
      FP32-stage, one persistent launch per stage, CUDA graph.
"""
from __future__ import annotations

import numpy as np

from . import TS_BC_DIRICHLET, TS_BC_NOOP, TS_F32_STAGE, TS_F64, TS_MODEL_WAVE, TS_RK4, WaveDesc

TS_F32_STAGE_DEFAULT = TS_F32_STAGE


def wave_desc(
    n,
    ngrow: int,
    *,
    periodic=(1, 1, 1),
    ko: float = 0.0,
    abl_thickness: int = 0,
    abl_max: float = 0.0,
    abl_profile: int = 2,
    bc: int = TS_BC_NOOP,
    bc_values=(0.0, 0.0),
    dt: float | None = None,
    cfl: float = 0.25,
    scheme: int = TS_RK4,
    precision: int = TS_F64,
    prob_lo=(0.0, 0.0, 0.0),
    prob_hi=(1.0, 1.0, 1.0),
    model: int = TS_MODEL_WAVE,
    block=(0, 0, 0),
    rtol: float = 0.0,
    atol: float = 0.0,
) -> WaveDesc:
    d = WaveDesc()
    n = (n, n, n) if np.isscalar(n) else tuple(n)
    d.n[:] = list(n)
    d.prob_lo[:] = list(prob_lo)
    d.prob_hi[:] = list(prob_hi)
    d.periodic[:] = [int(p) for p in periodic]
    d.ngrow = ngrow
    d.model = model
    d.ko_strength = ko
    d.abl_thickness = abl_thickness
    d.abl_max_strength = abl_max
    d.abl_profile = abl_profile
    d.bc = bc
    for q, v in enumerate(bc_values):
        d.bc_values[q] = v
    dx = (prob_hi[0] - prob_lo[0]) / n[0]
    d.dt = dt if dt is not None else cfl * dx
    d.scheme = scheme
    d.precision = precision
    d.c2 = None
    d.block[:] = list(block)
    d.rtol = rtol
    d.atol = atol
    return d


def c1_desc(precision: int = TS_F64) -> WaveDesc:
    return wave_desc(64, 2, ko=0.1, precision=precision)


def c1_pulses() -> np.ndarray:
    return np.array([[0, 1.0, 0.1, 0.5, 0.5, 0.5]], dtype=np.float64)


def c2_desc(precision: int = TS_F64, n: int = 256) -> WaveDesc:
    return wave_desc(
        n,
        4,
        periodic=(0, 0, 0),
        ko=0.2,
        abl_thickness=16 if n >= 64 else max(1, n // 8),
        abl_max=10.0,
        abl_profile=2,
        bc=TS_BC_DIRICHLET,
        bc_values=(0.0, 0.0),
        precision=precision,
    )


def c2_pulses(seed: int = 2024, npulses: int = 8) -> np.ndarray:
    rng = np.random.default_rng(seed)
    p = np.zeros((npulses, 6))
    p[:, 0] = 0
    p[:, 1] = rng.uniform(0.5, 1.0, npulses)
    p[:, 2] = rng.uniform(0.05, 0.15, npulses)
    p[:, 3:6] = rng.uniform(0.25, 0.75, (npulses, 3))
    return p


C1_STEPS = 100
C2_STEPS = 1000


C4_STEPS = 200


def c4_descs(precision: int = TS_F32_STAGE_DEFAULT, count: int = 512, seed: int = 4004) -> list[WaveDesc]:
    rng = np.random.default_rng(seed)
    edges = rng.choice(np.arange(16, 97, 8), size=count)
    return [wave_desc(int(n), 2, periodic=(1, 1, 1), precision=precision, dt=0.25 / int(n)) for n in edges]


def c4_pulses(count: int = 512, seed: int = 4005) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        a, w = rng.uniform(0.5, 1.0), rng.uniform(0.05, 0.2)
        c = rng.uniform(0.3, 0.7, 3)
        out.append(np.array([[0, a, w, *c]], dtype=np.float64))
    return out


C5_STEPS = 200
C5_CHECKPOINT_EVERY = 20


def c5_desc(n: int = 128, ngrow: int = 2) -> WaveDesc:
    """C5: 128^3 periodic unit cube, phi_t = pi, pi_t = c(x)^2 sum D2 phi + KO 0.1 (order ngrow), RK4 dt = 0.25 dx."""
    return wave_desc(n, ngrow, periodic=(1, 1, 1), ko=0.1)


def c5_speed(n: int = 128, seed: int = 5005, modes: int = 16, kmax: int = 4) -> np.ndarray:
    """c = 1 + 0.2 f / max|f|, f a sum of `modes` seeded Fourier modes with |k| <= kmax; (nz, ny, nx)."""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) + 0.5) / n
    z3, y3, x3 = np.meshgrid(x, x, x, indexing="ij")
    f = np.zeros((n, n, n))
    added = 0
    while added < modes:
        k = rng.integers(-kmax, kmax + 1, 3)
        if not k.any() or np.linalg.norm(k) > kmax:
            continue
        f += rng.normal() * np.cos(2 * np.pi * (k[0] * x3 + k[1] * y3 + k[2] * z3) + rng.uniform(0, 2 * np.pi))
        added += 1
    return 1.0 + 0.2 * f / np.abs(f).max()


def c5_pulse(n: int = 128, shift_cells: float = 0.0, amplitude: float = 1.0, width: float = 0.1) -> np.ndarray:
    """phi0 = A exp(-|x - c|^2 / w^2), c = (1/2 + shift dx, 1/2, 1/2); (nz, ny, nx)."""
    x = (np.arange(n) + 0.5) / n
    z3, y3, x3 = np.meshgrid(x, x, x, indexing="ij")
    cx = 0.5 + shift_cells / n
    return amplitude * np.exp(-((x3 - cx) ** 2 + (y3 - 0.5) ** 2 + (z3 - 0.5) ** 2) / width**2)


C3_STEPS = 500


def c3_desc(precision: int = TS_F32_STAGE_DEFAULT, n: int = 192) -> WaveDesc:
    """C3: tensorial wave system (h_ij, p_ij), n^3 periodic unit cube, ngrow 3, KO 0.1, RK4 dt = 0.25 dx."""
    from . import TS_MODEL_TENSOR_WAVE

    return wave_desc(n, 3, periodic=(1, 1, 1), ko=0.1, precision=precision, model=TS_MODEL_TENSOR_WAVE)


def c3_modes(seed: int = 3003, count: int = 32, kmax: int = 8) -> np.ndarray:
    """h_ij(0) = sum of `count` seeded Fourier modes (component, A ~ N(0, 0.01), integer k, |k| <= kmax, phase)."""
    rng = np.random.default_rng(seed)
    out = []
    while len(out) < count:
        k = rng.integers(-kmax, kmax + 1, 3)
        if not k.any() or np.linalg.norm(k) > kmax:
            continue
        out.append([rng.integers(0, 6), rng.normal(0.0, 0.01), *k, rng.uniform(0, 2 * np.pi)])
    return np.array(out, dtype=np.float64)
