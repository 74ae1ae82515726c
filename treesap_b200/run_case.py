"""Run one benchmark configuration through the C ABI and print its device time.

    python -m treesap_b200.run_case [--form f32|f64] [--n 256] [--steps 3] [--warmup 1] [--profile]

Used for profiling captures (e.g. `ncu ... python -m treesap_b200.run_case --form f64`):
C2-shaped workload (8th order, KO 0.2, absorbing layer, Dirichlet 0) at edge n.
--profile adds per-kernel device times (CUDA events around every launch) over the same steps.
"""
from __future__ import annotations

import argparse

from . import TS_F32_STAGE, TS_F64, TS_INIT_GAUSSIAN, Context, Integrator
from .configs import c2_desc, c2_pulses


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--form", choices=["f32", "f64"], default="f32")
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--profile", action="store_true")
    a = ap.parse_args()
    ctx = Context(0)
    it = Integrator(ctx, c2_desc(TS_F32_STAGE if a.form == "f32" else TS_F64, a.n))
    it.initialise(TS_INIT_GAUSSIAN, c2_pulses())
    it.step(a.warmup)
    it.step(a.steps)
    ctx.sync()
    ms, launches = it.last_step_timing()
    n3 = a.n**3
    print(f"form={a.form} n={a.n} steps={a.steps}: {ms / max(1, a.steps):.3f} ms/step, "
          f"{n3 * a.steps / (ms * 1e-3) / 1e9:.2f} G cell-updates/s, {launches} launches")
    if a.profile:
        counts, times = it.profile(a.steps)
        names = ["ghost fill"] + [f"stage {s}" for s in range(len(counts) - 1)]
        for name, c, t in zip(names, counts, times):
            if c:
                print(f"  {name:10s} {c:5d} launches  {1e3 * t / c:8.1f} us/launch")


if __name__ == "__main__":
    main()
