"""Loader of the golden fixtures in tests/golden/ (made by tests/golden/make_golden.py)."""
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden"


def names():
    return sorted(p.stem for p in GOLDEN.glob("*.npz"))


def load(name):
    z = np.load(GOLDEN / f"{name}.npz")
    d = {k[5:]: z[k] for k in z.files if k.startswith("desc_")}
    inp = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    return d, inp, int(z["nsteps"]), float(z["time"]), z["out"]


def ref_desc(d):
    from oracle import pyoracle

    r = pyoracle.RefDesc()
    r.n[:] = [int(v) for v in d["n"]]
    r.prob_lo[:] = [float(v) for v in d["prob_lo"]]
    r.prob_hi[:] = [float(v) for v in d["prob_hi"]]
    r.periodic[:] = [int(v) for v in d["periodic"]]
    r.ngrow = int(d["ngrow"])
    r.model = int(d["model"])
    r.ko_strength = float(d["ko_strength"])
    r.abl_thickness = int(d["abl_thickness"])
    r.abl_max_strength = float(d["abl_max_strength"])
    r.abl_profile = int(d["abl_profile"])
    r.bc = int(d["bc"])
    r.bc_values[:] = [float(v) for v in d["bc_values"]]
    r.dt = float(d["dt"])
    r.integrator = int(d["integrator"])
    r.block[:] = [int(v) for v in d["block"]]
    return r


def run_kwargs(inp):
    kw = {}
    if "state" in inp:
        kw["state"] = inp["state"]
    if "items" in inp:
        kw["items"] = inp["items"]
        kw["init_kind"] = int(inp["kind"]) if "kind" in inp else 1
    if "c2" in inp:
        kw["c2"] = inp["c2"]
    return kw
