"""Run the batched configuration (C4) through the C ABI and print its device time.

    python -m treesap_b200.run_batch [--count 512] [--steps 200] [--form f32|f64] [--autotune] [--no-graph]

512 periodic scalar-wave instances with cube edges 16..96 (ngrow 2, no KO), one Gaussian each,
advanced together: one persistent launch per RK4 stage, one ghost-fill launch per stage,
each step replayed from a CUDA graph.
"""
from __future__ import annotations

import argparse

from . import TS_F32_STAGE, TS_F64, TS_INIT_GAUSSIAN, Batch, Context
from .configs import C4_STEPS, c4_descs, c4_pulses


def run(ctx, count=512, steps=C4_STEPS, warmup=3, form="f32", autotune=True, graph=True, seed=4004):
    descs = c4_descs(TS_F32_STAGE if form == "f32" else TS_F64, count, seed)
    pulses = c4_pulses(count, seed + 1)
    b = Batch(ctx, descs)
    for i in range(count):
        b.initialise(i, TS_INIT_GAUSSIAN, pulses[i])
    shape = (0, 0)
    if autotune:
        shape = b.autotune(3)
    b.use_graph(graph)
    b.step(warmup)
    ctx.sync()
    b.step(steps)
    ctx.sync()
    ms, launches = b.last_step_timing()
    cells = sum(d.n[0] * d.n[1] * d.n[2] for d in descs)
    return {"batch": b, "descs": descs, "ms": ms, "launches": launches, "cells": cells, "shape": shape,
            "value": cells * steps / (ms * 1e-3)}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--steps", type=int, default=C4_STEPS)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--form", choices=["f32", "f64"], default="f32")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--no-graph", action="store_true")
    a = ap.parse_args()
    ctx = Context(0)
    r = run(ctx, a.count, a.steps, a.warmup, a.form, a.autotune, not a.no_graph)
    print(f"form={a.form} instances={a.count} cells={r['cells']} steps={a.steps}: {r['ms'] / a.steps:.3f} ms/step, "
          f"{r['value'] / 1e9:.2f} G cell-updates/s, {r['launches']} launches, shape(rows, zchunk)={r['shape']}")


if __name__ == "__main__":
    main()
