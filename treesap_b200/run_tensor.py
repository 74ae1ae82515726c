"""Run the tensorial wave configuration (C3) in both forms and print throughput and error.

    python -m treesap_b200.run_tensor [--n 192] [--steps 20] [--warmup 2]

192^3 periodic, 12 components (h_ij, p_ij as two symmetric-tensor aliases), 6th-order
stencils with mixed derivatives and the trace, KO 0.1, RK4 dt = 0.25 dx; h_ij(0) = 32 seeded
Fourier modes. Both forms start from the same state; the FP32-stage result is compared with
the FP64 one after warmup + steps steps.
"""
from __future__ import annotations

import argparse

import numpy as np

from . import TS_F32_STAGE, TS_F64, TS_INIT_FOURIER, Context, Integrator
from .configs import c3_desc, c3_modes


def run(ctx, n=192, steps=20, warmup=2):
    res = {}
    states = {}
    for name, prec in (("f32", TS_F32_STAGE), ("f64", TS_F64)):
        it = Integrator(ctx, c3_desc(prec, n))
        it.initialise(TS_INIT_FOURIER, c3_modes())
        it.step(warmup)
        ctx.sync()
        it.step(steps)
        ctx.sync()
        ms, launches = it.last_step_timing()
        res[name] = {"value": n**3 * steps / (ms * 1e-3), "ms_per_step": ms / steps, "launches": launches}
        states[name] = it.get_state()
        it.close()
    d = states["f32"] - states["f64"]
    res["error_f32_vs_f64"] = {"steps": warmup + steps,
                               "maxnorm_rel": float(np.abs(d).max() / np.abs(states["f64"]).max()),
                               "l2_rel": float(np.linalg.norm(d) / np.linalg.norm(states["f64"]))}
    return res


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=192)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=2)
    a = ap.parse_args()
    ctx = Context(0)
    print(run(ctx, a.n, a.steps, a.warmup))


if __name__ == "__main__":
    main()
