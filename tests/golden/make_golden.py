"""Generates tests/golden/*.npz from the reference's own integrators.

    python tests/golden/make_golden.py

Every case runs oracle/_ref/libtsref.so, i.e. the reference headers (src/treesap/**) compiled
unchanged against the host AMReX-API shim in oracle/amrex_host/, on a small seeded input and
stores the descriptor, the input and the final valid state. The reference publishes no golden
vectors of its own, so these fixtures (plus the analytic known-answer tests in
tests/test_kat.py) pin the CPU restatement oracle/ts_oracle.c and, through it, the GPU path.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import pyoracle  # noqa: E402

OUT = Path(__file__).resolve().parent


def desc(n, ngrow, **kw):
    d = pyoracle.RefDesc()
    d.n[:] = list(n)
    d.prob_lo[:] = list(kw.get("lo", (0.0, 0.0, 0.0)))
    d.prob_hi[:] = list(kw.get("hi", (1.0, 1.0, 1.0)))
    d.periodic[:] = list(kw.get("periodic", (1, 1, 1)))
    d.ngrow = ngrow
    d.model = kw.get("model", 0)
    d.ko_strength = kw.get("ko", 0.0)
    d.abl_thickness = kw.get("abl", 0)
    d.abl_max_strength = kw.get("abl_max", 0.0)
    d.abl_profile = kw.get("abl_profile", 2)
    d.bc = kw.get("bc", 0)
    for q, v in enumerate(kw.get("bc_values", ())):
        d.bc_values[q] = v
    d.dt = kw.get("dt", 0.2 / max(n))
    d.integrator = kw.get("integrator", 1)
    d.block[:] = list(kw.get("block", (0, 0, 0)))
    return d


def desc_dict(d) -> dict:
    return {
        "n": np.array(d.n[:], dtype=np.int64),
        "prob_lo": np.array(d.prob_lo[:]),
        "prob_hi": np.array(d.prob_hi[:]),
        "periodic": np.array(d.periodic[:], dtype=np.int64),
        "ngrow": np.int64(d.ngrow),
        "model": np.int64(d.model),
        "ko_strength": np.float64(d.ko_strength),
        "abl_thickness": np.int64(d.abl_thickness),
        "abl_max_strength": np.float64(d.abl_max_strength),
        "abl_profile": np.int64(d.abl_profile),
        "bc": np.int64(d.bc),
        "bc_values": np.array(d.bc_values[:]),
        "dt": np.float64(d.dt),
        "integrator": np.int64(d.integrator),
        "block": np.array(d.block[:], dtype=np.int64),
    }


def random_state(rng, ncomp, n):
    return rng.standard_normal((ncomp, n[2], n[1], n[0]))


def cases():
    rng = np.random.default_rng(20241203)
    n = (10, 9, 11)
    for g in (1, 2, 3, 4):
        for ko in (0.0, 0.1):
            yield f"wave_periodic_g{g}_ko{int(ko * 10)}", desc(n, g, ko=ko), dict(state=random_state(rng, 2, n)), 3
    for g in (2, 4):
        yield (f"wave_dirichlet_g{g}", desc(n, g, periodic=(1, 0, 0), bc=1, bc_values=(0.3, -0.2), ko=0.15,
                                           lo=(-1, 0, 0.5), hi=(1, 1, 2)), dict(state=random_state(rng, 2, n)), 3)
        yield (f"wave_abl_quadratic_g{g}", desc(n, g, periodic=(0, 0, 0), abl=3, abl_max=7.0, bc_values=(0.1, 0.0),
                                                ko=0.2), dict(state=random_state(rng, 2, n)), 3)
        yield (f"wave_euler_abl_linear_g{g}", desc(n, g, periodic=(0, 0, 0), abl=2, abl_max=5.0, abl_profile=1,
                                                   integrator=0), dict(state=random_state(rng, 2, n)), 4)
    yield ("wave_blocks_g2", desc((12, 10, 9), 2, ko=0.1, block=(5, 4, 4)),
           dict(state=random_state(rng, 2, (12, 10, 9))), 3)
    c2 = (1.0 + 0.2 * rng.uniform(-1, 1, (n[2], n[1], n[0]))) ** 2
    yield "wave_speed_g2", desc(n, 2, ko=0.1), dict(state=random_state(rng, 2, n), c2=c2), 3
    yield ("wave_gaussian_init_g4", desc((16, 14, 12), 4, periodic=(0, 0, 0), bc=1),
           dict(items=np.array([[0, 0.8, 0.15, 0.5, 0.45, 0.55], [1, 0.3, 0.2, 0.4, 0.5, 0.5]])), 2)
    m = [[c, rng.normal(0, 0.01), rng.integers(-3, 4), rng.integers(-3, 4), rng.integers(-3, 4),
          rng.uniform(0, 2 * np.pi)] for c in range(6) for _ in range(3)]
    for g in (2, 3):
        yield f"tensor_periodic_g{g}", desc((8, 8, 8), g, model=1, ko=0.1), dict(items=np.array(m, dtype=float),
                                                                             kind=2), 2


def main():
    orc = pyoracle.Oracle("ref")
    for name, d, inp, nsteps in cases():
        kw = {}
        if "state" in inp:
            kw["state"] = inp["state"]
        if "items" in inp:
            kw["items"] = inp["items"]
            kw["init_kind"] = inp.get("kind", pyoracle.INIT_GAUSSIAN)
        if "c2" in inp:
            kw["c2"] = inp["c2"]
        out, _, t = orc.run(d, nsteps, **kw)
        arrays = {f"desc_{k}": v for k, v in desc_dict(d).items()}
        arrays.update({f"in_{k}": np.asarray(v) for k, v in inp.items()})
        arrays["nsteps"] = np.int64(nsteps)
        arrays["time"] = np.float64(t)
        arrays["out"] = out
        np.savez_compressed(OUT / f"{name}.npz", **arrays)
        print(f"{name}: {out.shape} max|u| = {np.abs(out).max():.3e}")


if __name__ == "__main__":
    main()
