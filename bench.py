#!/usr/bin/env python3
"""Benchmark of the single-level RK4 path on the 256^3 8th-order wave problem (C2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload (seeded synthetic data, no dataset): 256^3 cells on the unit cube, scalar wave
{phi, pi}, 8th-order centred stencils (ngrow 4), Kreiss-Oliger 0.2, absorbing layer of 16
cells (profile s^2, max 10/L, targets 0, Dirichlet-0 ghosts), RK4 with dt = 0.25 dx;
phi0 = 8 Gaussian pulses (A ~ U[0.5,1], w ~ U[0.05,0.15], c ~ U[0.25,0.75]^3, seed 2024).
A bench step is one RK4 time step over the whole grid. Both forms run W + K steps from the
same initial state: the FP32-stage form (the headline `value`) and the FP64 plain form;
after the run the FP32-stage result is compared with the FP64 one (max-norm, L2).

Timing: K steps bracketed by barrier + synchronize, CUDA events on the library's stream,
max over ranks. Every field (268 MB) is larger than L2 (126 MB), so no L2 flush is needed
between steps. `e2e` times the C ABI call ts_integrator_run (pinned host state in -> 20
steps -> host state out) with the host<->device copies inside the timed region.
The line also carries `batched`: the C4 workload (512 periodic instances, edges 16..96) through
ts_batch_* (autotuned launch shape, one persistent launch per stage, CUDA graph), 200 steps, and
`adjoint`: the C5 loss + gradient through ts_adjoint_* (seconds, and the largest relative
difference to central finite differences over 32 random directions of phi0 and of c), and
`tensor`: C3 (192^3, 12 components) for a few steps of each form.
For N > 1 the ranks share one 256 x 256 x 256N domain, one 256^3 z slab per GPU (weak
scaling), exchanging their boundary planes every RK4 stage over NCCL (treesap_b200/slabs.py).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "RK4 cell-updates/s @256^3: FP32 vs FP64 at err<=1e-6; % of HBM peak"
UNIT = "cell-updates/s"
N = 256
E2E_CHUNK = 20  # steps per end-to-end call (the plot-export cadence of the reference's driver)
BATCH_STEPS = 200  # C4 step count
TENSOR_STEPS = 3  # C3 steps per form (about 1 s per step)
# Algorithmic HBM bytes per cell and launch (2 components, valid cells only, ghost fills excluded).
ALG_BYTES = {
    # FP32-stage per component: R u8 W k0 8 W u_p 8 | R k0 8 W d1 4 | R d1 4 W d2 4 | R d2 4, d1 4, u_p 8 W u 8
    "f32": {1: 48, 2: 24, 3: 16, 4: 48},
    "f64": {1: 48, 2: 80, 3: 80, 4: 48},  # reference register scheme: 3, 5, 5, 3 words per component
}
KERNEL_NAMES = {0: "ghost_fill", 1: "stage_kernel[s=0]", 2: "stage_kernel[s=1]", 3: "stage_kernel[s=2]",
                4: "stage_kernel[s=3]"}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Dist:
    """Barriers and max-reductions across ranks (torch.distributed over gloo; no-op for one rank)."""

    def __init__(self, world, local_rank=0):
        self.world = world
        self.dist = None
        if world > 1:
            import datetime

            import torch
            import torch.distributed as dist

            # host tensors (barriers, timings) over gloo, device tensors (slab planes) over NCCL;
            # gloo alone on a host without a GPU (the host-side logic runs there too)
            backend = "gloo"
            if torch.cuda.is_available():
                torch.cuda.set_device(local_rank)
                backend = "cpu:gloo,cuda:nccl"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.dist = dist

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if not self.dist:
            return v
        import torch

        t = torch.tensor([v], dtype=torch.float64)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.lines, self.proc = device, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i", str(self.device),
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def hbm_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback"


def traffic_from_profiles(key: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary (null when absent)."""
    try:
        t = json.loads((ROOT / "profiles" / "dram_traffic_c2_256.json").read_text())
        return t.get("bytes", {}).get(key)
    except (OSError, ValueError):
        return None


def cpu_baseline(desc, pulses, budget_s=15.0):
    """The reference's own headers (oracle/_ref) on the host cores: same workload, bounded step count."""
    from oracle import pyoracle

    which = "ref" if pyoracle.available("ref") else "port"
    orc = pyoracle.Oracle(which)
    _, t1, _ = orc.run(desc, 1, items=pulses)
    nsteps = int(max(1, min(10, budget_s / max(t1, 1e-3))))
    state, secs, _ = orc.run(desc, nsteps, items=pulses)
    ncell = desc.n[0] * desc.n[1] * desc.n[2]
    cpu_baseline.last = (which, nsteps, state)  # kept for the parity check of the bench line
    return {
        "value": ncell * nsteps / secs,
        "unit": UNIT,
        "cores": orc.threads,
        "kind": "reference" if which == "ref" else "port",
        "sample": f"{nsteps} RK4 steps of the full 256^3 workload (FP64) on {orc.threads} host threads "
                  f"({pyoracle.cpu_model()}, {pyoracle.host_cores()} cores visible)",
    }


def run_reference(args, rank, world):
    """--impl reference: the reference's CPU implementation (oracle/_ref), rank 0 only."""
    if rank != 0:
        return
    from oracle import pyoracle
    from treesap_b200.configs import c2_desc, c2_pulses

    if not pyoracle.available("ref"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtsref.so (the reference headers "
                          "built against the host AMReX-API shim) is not built"}))
        return
    orc = pyoracle.Oracle("ref")
    pulses = c2_pulses()
    # a bounded sample of the workload per step: the full 256 x 256 cross-section, nz planes
    probe = c2_desc(n=N)
    probe.n[2] = 32
    probe.prob_hi[2] = 32 / N
    _, t32, _ = orc.run(probe, 1, items=pulses)
    budget = 150.0
    nz = int(np.clip(32 * budget / max(1e-3, t32 * (args.steps + args.warmup + 1)), 16, N))
    d = c2_desc(n=N)
    d.n[2] = nz
    d.prob_hi[2] = nz / N
    orc.run(d, args.warmup, items=pulses)
    _, secs, _ = orc.run(d, args.steps, items=pulses)
    ncell = N * N * nz
    v = ncell * args.steps / secs
    sample = (f"each step: one RK4 step of a 256 x 256 x {nz} slab of the 256^3 workload (same stencils, KO, "
              f"absorbing layer, Dirichlet ghosts), {orc.threads} host threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "C2 256^3 scalar wave, 8th order, KO 0.2, absorbing layer 16 (s^2, max 10), "
                   "Dirichlet 0, RK4 dt=0.25dx", "grid": [N, N, nz], "sample": "z slab"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": orc.threads, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def timed_form(ts, ctx, dist, precision, pulses, args, local_rank):
    from treesap_b200 import TS_INIT_GAUSSIAN, Integrator
    from treesap_b200.configs import c2_desc

    it = Integrator(ctx, c2_desc(precision, N))
    it.initialise(TS_INIT_GAUSSIAN, pulses)
    it.step(args.warmup)
    ctx.sync()
    dist.barrier()
    with ClockSampler(local_rank) as clk:
        it.step(args.steps)
        ctx.sync()
    dist.barrier()
    ms, launches = it.last_step_timing()
    return it, ms, launches, clk.summary()


def run_sharded(args, rank, world, local_rank):
    """N > 1: one domain of 256 x 256 x 256N cells (8 seeded pulses scaled along z) split into N
    z slabs, one per GPU (weak scaling: every GPU holds a 256^3 slab); per RK4 stage each rank
    exchanges its ngrow boundary planes with its neighbours over NCCL (treesap_b200.slabs)."""
    import torch

    from treesap_b200 import TS_F32_STAGE, TS_F64, TS_INIT_GAUSSIAN, Context
    from treesap_b200.configs import c2_desc, c2_pulses
    from treesap_b200.slabs import SlabDomain, TorchComm

    dist = Dist(world, local_rank)
    ctx = Context(local_rank)
    ncell = N * N * N  # cells per rank
    pulses = c2_pulses()
    pulses[:, 5] = (pulses[:, 5] + np.arange(len(pulses)) % world) / world  # spread the pulses over the slabs
    res = {}
    for name, prec in (("f32", TS_F32_STAGE), ("f64", TS_F64)):
        desc = c2_desc(prec, N)
        desc.n[2] = N * world
        desc.prob_hi[2] = float(world)
        dom = SlabDomain(desc, rank, world, TorchComm(ctx.stream), ctx=ctx)
        dom.slab.initialise(TS_INIT_GAUSSIAN, pulses)
        dom.step(args.warmup)
        ctx.sync()
        dist.barrier()
        stream = torch.cuda.ExternalStream(ctx.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as clk:
            ev0.record(stream)
            dom.step(args.steps)
            ev1.record(stream)
            ev1.synchronize()
        dist.barrier()
        ms = dist.max(ev0.elapsed_time(ev1))
        res[name] = {"ms": ms, "value": world * ncell * args.steps / (ms * 1e-3), "clocks": clk.summary(), "dom": dom}

    # end to end: host state in -> steps -> host state out, per rank (its slab), FP32-stage form
    dom = res["f32"]["dom"]
    host = dom.slab.get_state()
    dist.barrier()
    t0 = time.perf_counter()
    dom.slab.set_state(host)
    dom.step(E2E_CHUNK)
    out = dom.slab.get_state()
    secs = dist.max(time.perf_counter() - t0)
    e2e = {"value": world * ncell * E2E_CHUNK / secs, "unit": UNIT, "h2d_bytes_per_step": world * host.nbytes / E2E_CHUNK,
           "d2h_bytes_per_step": world * out.nbytes / E2E_CHUNK,
           "call": f"per rank: slab set_state(host) -> {E2E_CHUNK} sharded steps -> get_state(host), FP32-stage form"}
    for r in res.values():
        r["dom"].slab.close()
    if rank == 0:
        f32, f64 = res["f32"], res["f64"]
        line = {
            "metric": METRIC, "value": f32["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": f32["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-stage+f64-state", "data": "synthetic",
            "config": {"workload": "C2 scalar wave, 8th-order (ngrow 4), KO 0.2, absorbing layer 16 cells, Dirichlet 0, "
                       "RK4 dt=0.25dx, 8 seeded pulses; one 256 x 256 x 256N domain in N z slabs",
                       "grid": [N, N, N * world], "form": "FP32-stage RK4 (FP64 state and final combination)",
                       "l2": "no flush: every field exceeds L2 (126 MB)",
                       "parallelism": f"z slabs x{world}, NCCL halo exchange per stage"},
            "fp64": {"value": f64["value"], "ms_per_step": f64["ms"] / args.steps},
            "speedup_f32_over_f64": f32["value"] / f64["value"],
            "cpu_baseline": None, "e2e": e2e,
            # per stage and rank: the stage kernel and one halo copy per exchanged face (the static
            # Dirichlet ghost cells are filled once per buffer, before the timed steps)
            "gpu_launches": args.steps * 4 * (1 + (dom.lo is not None) + (dom.hi is not None)),
            "clocks": {k: f32["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(line))
    ctx.close()
    dist.close()


def run_b200(args, rank, world, local_rank):
    from treesap_b200 import TS_F32_STAGE, TS_F64, Context
    from treesap_b200.configs import c2_desc, c2_pulses

    dist = Dist(world)
    ctx = Context(local_rank)
    pulses = c2_pulses()
    ncell = N**3
    res = {}
    for name, prec in (("f32", TS_F32_STAGE), ("f64", TS_F64)):
        it, ms, launches, clocks = timed_form(None, ctx, dist, prec, pulses, args, local_rank)
        ms_max = dist.max(ms)
        res[name] = {"it": it, "ms": ms_max, "launches": launches, "clocks": clocks,
                     "value": world * ncell * args.steps / (ms_max * 1e-3)}

    # accuracy of the FP32-stage form against the FP64 form after W + K steps from the same state
    a32 = res["f32"]["it"].get_state()
    a64 = res["f64"]["it"].get_state()
    diff = a32 - a64
    err = {"steps": args.warmup + args.steps,
           "maxnorm_abs": float(np.abs(diff).max()),
           "maxnorm_rel": float(np.abs(diff).max() / np.abs(a64).max()),
           "l2_rel": float(np.linalg.norm(diff) / np.linalg.norm(a64)),
           "per_component_maxnorm_abs": [float(np.abs(diff[c]).max()) for c in range(diff.shape[0])]}

    # per-kernel device times (CUDA events around every launch) over a further stretch of steps
    prof_steps = min(args.steps, 50)
    peak, peak_kind = hbm_peak()
    kernels = {}
    for name in ("f32", "f64"):
        n, ms = res[name]["it"].profile(prof_steps)
        per = {}
        for cls in range(5):
            if n[cls] == 0:
                continue
            avg = ms[cls] / n[cls]
            e = {"launches": n[cls], "avg_ms": avg, "share": ms[cls] / sum(ms)}
            if cls in ALG_BYTES[name]:
                alg = ALG_BYTES[name][cls] * ncell
                e["alg_bytes"] = alg
                e["achieved_gbs"] = alg / (avg * 1e-3) / 1e9
            per[KERNEL_NAMES[cls]] = e
        kernels[name] = per
    stage = {k: v for k, v in kernels["f32"].items() if "alg_bytes" in v}
    dom_name, dom = max(stage.items(), key=lambda kv: kv[1]["share"])
    traffic = traffic_from_profiles(f"f32/{dom_name}")
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": dom["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": dom["achieved_gbs"] / peak, "traffic": traffic, "peak_kind": peak_kind,
                "alg_bytes_per_launch": dom["alg_bytes"], "avg_launch_ms": dom["avg_ms"]}
    step_bytes = {k: sum(ALG_BYTES[k].values()) * ncell for k in ALG_BYTES}
    step_frac = {k: step_bytes[k] / (res[k]["ms"] / args.steps * 1e-3) / 1e9 / peak for k in ("f32", "f64")}

    # end to end through the C ABI with pinned host buffers
    e2e = None
    try:
        import torch

        pin_in = torch.empty((2, N, N, N), dtype=torch.float64, pin_memory=True).numpy()
        pin_out = torch.empty((2, N, N, N), dtype=torch.float64, pin_memory=True).numpy()
        pin_in[...] = a64
        it = res["f32"]["it"]
        it.run(pin_in, E2E_CHUNK, pin_out)  # warm-up call
        ncalls = max(3, args.steps // 200)
        torch.cuda.set_device(local_rank)
        stream = torch.cuda.ExternalStream(ctx.stream)  # events on the library's own stream
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        dist.barrier()
        ev0.record(stream)
        for _ in range(ncalls):
            it.run(pin_in, E2E_CHUNK, pin_out)
        ev1.record(stream)
        ev1.synchronize()
        secs = dist.max(ev0.elapsed_time(ev1) * 1e-3)
        bytes_io = pin_in.nbytes
        e2e = {"value": world * ncell * E2E_CHUNK * ncalls / secs, "unit": UNIT,
               "h2d_bytes_per_step": bytes_io / E2E_CHUNK, "d2h_bytes_per_step": bytes_io / E2E_CHUNK,
               "call": f"ts_integrator_run(host_in, {E2E_CHUNK} steps, host_out), FP32-stage form, pinned host "
                       f"buffers; {ncalls} calls timed"}
    except Exception as ex:  # noqa: BLE001 - reported in the line
        e2e = {"value": None, "unit": UNIT, "error": str(ex)}

    cpu = cpu_baseline(c2_desc(TS_F64, N), pulses) if (rank == 0 and world == 1) else None

    # parity at the benchmarked size: the GPU FP64 form against the reference build, the same
    # steps from the same pulses as the CPU baseline's sample
    parity = None
    if cpu is not None:
        from treesap_b200 import TS_INIT_GAUSSIAN, Integrator

        which, nsteps, want = cpu_baseline.last
        chk = Integrator(ctx, c2_desc(TS_F64, N))
        chk.initialise(TS_INIT_GAUSSIAN, pulses)
        chk.step(nsteps)
        got = chk.get_state()
        chk.close()
        d = got - want
        parity = {"against": "reference build (oracle/_ref)" if which == "ref" else "oracle port", "form": "FP64",
                  "grid": [N, N, N], "steps": nsteps, "maxnorm_rel": float(np.abs(d).max() / np.abs(want).max()),
                  "l2_rel": float(np.linalg.norm(d) / np.linalg.norm(want)), "tolerance": 1e-12}
        parity["ok"] = parity["maxnorm_rel"] <= 1e-12

    # batched form (C4): 512 periodic instances, one persistent launch per stage, CUDA graph
    batched = None
    for r in res.values():
        r["it"].close()  # free the 256^3 fields first
    try:
        from treesap_b200.run_batch import run as run_batch

        dist.barrier()
        b = run_batch(ctx, steps=BATCH_STEPS, warmup=3, form="f32", autotune=True, graph=True)
        ms_b = dist.max(b["ms"])
        vb = world * b["cells"] * BATCH_STEPS / (ms_b * 1e-3)
        batched = {"workload": "C4: 512 periodic scalar-wave instances, edges U{16,24,...,96}, ngrow 2, no KO, "
                               "RK4 dt=0.25/n, one Gaussian each, FP32-stage", "value": vb, "unit": UNIT,
                   "steps": BATCH_STEPS, "ms_per_step": ms_b / BATCH_STEPS, "cells": b["cells"],
                   "launches_per_step": b["launches"] / BATCH_STEPS, "launch_shape_rows_zchunk": list(b["shape"]),
                   "hbm_frac_of_step": sum(ALG_BYTES["f32"].values()) * vb / world / 1e9 / peak}
        b["batch"].close()
    except Exception as ex:  # noqa: BLE001 - reported in the line
        batched = {"value": None, "error": str(ex)}

    # tensor model (C3): a few steps of each form (the 12-component kernels take tens of ms per step)
    tensor = None
    try:
        from treesap_b200.run_tensor import run as run_tensor

        r = run_tensor(ctx, steps=TENSOR_STEPS, warmup=1)
        tensor = {"workload": "C3: 192^3 periodic tensorial wave (h_ij, p_ij; 12 components), ngrow 3, KO 0.1, "
                              "RK4 dt=0.25dx, 32 seeded Fourier modes", "steps": TENSOR_STEPS,
                  "fp32_stage": r["f32"], "fp64": r["f64"], "error_f32_vs_f64": r["error_f32_vs_f64"]}
    except Exception as ex:  # noqa: BLE001 - reported in the line
        tensor = {"error": str(ex)}

    # discrete adjoint (C5): loss + gradient time and central-difference agreement
    adjoint = None
    try:
        from treesap_b200.run_adjoint import run as run_adjoint

        a = run_adjoint(ctx)
        adjoint = {"workload": "C5: 128^3 periodic variable-speed wave, ngrow 2, KO 0.1, RK4 200 steps, checkpoints "
                               "every 20, J = 1/2 sum (phi(T) - phi_target)^2, FP64",
                   "gradient_seconds": a["gradient_s"], "forward_seconds": a["forward_s"],
                   "gradient_over_forward": a["gradient_s"] / a["forward_s"],
                   "fd_directions": a["directions"], "fd_rel_err_max_phi0": a["fd_rel_max_phi0"],
                   "fd_rel_err_max_c": a["fd_rel_max_c"], "tolerance": 1e-5,
                   "fp32_stage": {"state_gradient_seconds": a["fp32_stage_state_gradient_s"],
                                  "gradient_seconds": a["fp32_stage_gradient_s"],
                                  "grad_phi0_maxnorm_rel_vs_fp64": a["fp32_stage_grad_phi0_rel_vs_fp64"],
                                  "grad_c_maxnorm_rel_vs_fp64": a["fp32_stage_grad_c_rel_vs_fp64"],
                                  "fd_rel_err_max_c": a["fp32_stage_fd_rel_max_c"],
                                  "loss_rel_vs_fp64": a["fp32_stage_loss_rel_vs_fp64"]}}
    except Exception as ex:  # noqa: BLE001 - reported in the line
        adjoint = {"error": str(ex)}

    if rank == 0:
        f32, f64 = res["f32"], res["f64"]
        line = {
            "metric": METRIC, "value": f32["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": f32["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32-stage+f64-state", "data": "synthetic",
            "config": {"workload": "C2 256^3 scalar wave, 8th-order (ngrow 4), KO 0.2, absorbing layer 16 cells "
                       "(s^2, max 10/L, target 0, Dirichlet-0 ghosts), RK4 dt=0.25dx, 8 seeded Gaussian pulses",
                       "grid": [N, N, N], "form": "FP32-stage RK4 (FP64 state and final combination)",
                       "l2": "no flush: every field (268 MB) exceeds L2 (126 MB)",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "fp64": {"value": f64["value"], "ms_per_step": f64["ms"] / args.steps,
                     "hbm_frac_of_step": step_frac["f64"], "alg_bytes_per_cell_update": sum(ALG_BYTES["f64"].values())},
            "fp32_stage": {"value": f32["value"], "hbm_frac_of_step": step_frac["f32"],
                           "alg_bytes_per_cell_update": sum(ALG_BYTES["f32"].values())},
            "speedup_f32_over_f64": f32["value"] / f64["value"],
            "error_f32_vs_f64": err,
            "roofline": roofline,
            "kernels": kernels,
            "cpu_baseline": cpu,
            "parity": parity,
            "e2e": e2e,
            "gpu_launches": int(f32["launches"]),
            "clocks": {k: f32["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "clocks_fp64_run": {k: f64["clocks"][k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "batched": batched,
            "adjoint": adjoint,
            "tensor": tensor,
        }
        print(json.dumps(line))
    ctx.close()
    dist.close()
    if parity is not None and not parity["ok"]:
        sys.exit(f"parity failure at {N}^3: GPU FP64 vs reference relative max-norm {parity['maxnorm_rel']:.3e}")


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    rank, world, local_rank = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        run_sharded(args, rank, world, local_rank)
        return
    run_b200(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
