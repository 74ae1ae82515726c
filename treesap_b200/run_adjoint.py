"""Run the adjoint configuration (C5) and check it against central finite differences.

    python -m treesap_b200.run_adjoint [--n 128] [--steps 200] [--every 20] [--directions 32]

128^3 periodic variable-speed wave (c = 1 + 0.2 f / max|f|, 16 Fourier modes, |k| <= 4),
4th-order stencils, KO 0.1, RK4 200 steps; loss J = 1/2 sum (phi(T) - phi_target)^2 with
phi_target from a forward run of the pulse shifted by 2 cells and scaled by 1.05. Prints the
time of one loss+gradient evaluation and, per random unit direction v of phi0 and of c, the
relative difference between <grad, v> and (J(p + eps v) - J(p - eps v)) / (2 eps); then the
FP32-stage form: the time of J + state gradient and of J + state and speed gradients, their
max-norm differences to the FP64 gradients, and the speed gradient against the same central
differences (of the FP64 loss).
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import Adjoint, Context
from .configs import C5_CHECKPOINT_EVERY, C5_STEPS, c5_desc, c5_pulse, c5_speed


def run(ctx, n=128, steps=C5_STEPS, every=C5_CHECKPOINT_EVERY, directions=32, seed=55):
    d = c5_desc(n)
    c = c5_speed(n)
    phi0 = c5_pulse(n)
    pi0 = np.zeros_like(phi0)
    adj = Adjoint(ctx, d, every)
    target, _ = adj.forward(c5_pulse(n, shift_cells=2, amplitude=1.05), pi0, c, steps)
    adj.gradient(phi0, pi0, c, steps, target)  # warm-up
    t0 = time.perf_counter()
    loss, gphi, gpi, gc = adj.gradient(phi0, pi0, c, steps, target)
    t_grad = time.perf_counter() - t0
    t0 = time.perf_counter()
    adj.forward(phi0, pi0, c, steps)
    t_fwd = time.perf_counter() - t0

    def J(p, c_):
        phiT, _ = adj.forward(p, pi0, c_, steps)
        return 0.5 * float(np.sum((phiT - target) ** 2))

    # FP32-stage form: state gradient alone, then state and speed gradients
    adj.gradient_f32(phi0, pi0, c, steps, target, speed=False)  # warm-up
    t0 = time.perf_counter()
    adj.gradient_f32(phi0, pi0, c, steps, target, speed=False)
    t_state32 = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss32, gphi32, _, gc32 = adj.gradient_f32(phi0, pi0, c, steps, target)
    t_grad32 = time.perf_counter() - t0

    rng = np.random.default_rng(seed)
    rel = {"phi0": [], "c": [], "c32": []}
    for _ in range(directions):
        v = rng.standard_normal(phi0.shape)
        v /= np.linalg.norm(v)
        for name, g, eps in (("phi0", gphi, 1e-3), ("c", gc, 1e-5)):
            if name == "phi0":
                fd = (J(phi0 + eps * v, c) - J(phi0 - eps * v, c)) / (2 * eps)
            else:
                fd = (J(phi0, c + eps * v) - J(phi0, c - eps * v)) / (2 * eps)
                ad32 = float(np.sum(gc32 * v))
                rel["c32"].append(abs(fd - ad32) / abs(ad32))
            ad = float(np.sum(g * v))
            rel[name].append(abs(fd - ad) / abs(ad))
    adj.close()

    def relmax(a, b):
        return float(np.abs(a - b).max() / np.abs(b).max())

    return {"loss": loss, "cells": n**3, "steps": steps, "checkpoint_every": every, "gradient_s": t_grad,
            "forward_s": t_fwd, "fd_rel_max_phi0": max(rel["phi0"]), "fd_rel_max_c": max(rel["c"]),
            "directions": directions, "fp32_stage_state_gradient_s": t_state32,
            "fp32_stage_gradient_s": t_grad32,
            "fp32_stage_grad_phi0_rel_vs_fp64": relmax(gphi32, gphi),
            "fp32_stage_grad_c_rel_vs_fp64": relmax(gc32, gc),
            "fp32_stage_fd_rel_max_c": max(rel["c32"]),
            "fp32_stage_loss_rel_vs_fp64": abs(loss32 - loss) / abs(loss)}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--steps", type=int, default=C5_STEPS)
    ap.add_argument("--every", type=int, default=C5_CHECKPOINT_EVERY)
    ap.add_argument("--directions", type=int, default=32)
    a = ap.parse_args()
    ctx = Context(0)
    r = run(ctx, a.n, a.steps, a.every, a.directions)
    print(r)


if __name__ == "__main__":
    main()
