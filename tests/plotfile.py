"""Reader of single-level AMReX plotfiles (HyperCLaw-V1.1 header, VisMF Cell_H, FAB data files),
following the documented on-disk layout; used by the exporter tests."""
import re
from pathlib import Path

import numpy as np


def _floats(line):
    return [float(v) for v in line.split()]


def read_plotfile(d):
    d = Path(d)
    h = (d / "Header").read_text().split("\n")
    assert h[0] == "HyperCLaw-V1.1", h[0]
    ncomp = int(h[1])
    names = h[2:2 + ncomp]
    i = 2 + ncomp
    out = {"names": names, "dim": int(h[i]), "time": float(h[i + 1]), "finest_level": int(h[i + 2]),
           "prob_lo": _floats(h[i + 3]), "prob_hi": _floats(h[i + 4])}
    assert h[i + 5] == ""  # no refinement ratios for a single level
    m = re.fullmatch(r"\(\((-?\d+),(-?\d+),(-?\d+)\) \((-?\d+),(-?\d+),(-?\d+)\) \(0,0,0\)\)", h[i + 6])
    lo, hi = [int(v) for v in m.groups()[:3]], [int(v) for v in m.groups()[3:]]
    out["n"] = [hi[a] - lo[a] + 1 for a in range(3)]
    out["level_step"] = int(h[i + 7])
    out["dx"] = _floats(h[i + 8])
    out["coord"], out["bwidth"] = int(h[i + 9]), int(h[i + 10])
    lev = h[i + 11].split()
    assert lev[0] == "0" and lev[1] == "1"
    out["step"] = int(h[i + 12])
    out["grid_phys"] = [_floats(h[i + 13 + a]) for a in range(3)]
    assert h[i + 16] == "Level_0/Cell"
    ch = (d / "Level_0" / "Cell_H").read_text().split("\n")
    assert ch[2] == str(ncomp) and ch[3] == "0"
    fod = [line for line in ch if line.startswith("FabOnDisk:")]
    assert len(fod) == 1
    _, fname, offset = fod[0].split()
    k = ch.index(fod[0])
    assert ch[k + 2] == f"1,{ncomp}"
    out["min"] = [float(v) for v in ch[k + 3].rstrip(",").split(",")]
    assert ch[k + 5] == f"1,{ncomp}"
    out["max"] = [float(v) for v in ch[k + 6].rstrip(",").split(",")]
    raw = (d / "Level_0" / fname).read_bytes()[int(offset):]
    nl = raw.index(b"\n")
    fab = raw[:nl].decode()
    assert fab.startswith("FAB ((8, (64 11 52 0 1 12 0 1023)),(8, (8 7 6 5 4 3 2 1)))"), fab
    assert fab.endswith(f" {ncomp}")
    n = out["n"]
    out["data"] = np.frombuffer(raw[nl + 1:], dtype="<f8", count=ncomp * n[0] * n[1] * n[2]).reshape(
        ncomp, n[2], n[1], n[0])
    return out
