"""ctypes binding of the CPU oracles (test infrastructure only; see tsref.h).

    ref     oracle/_ref/libtsref.so       the reference's own headers built unchanged
    port    oracle/_build/libtsoracle.so  plain-C restatement (ts_oracle.c)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arms use this
module, as the checker or the timed CPU baseline. Both libraries are built by
`make -C oracle` (the reference one only where the reference sources exist).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_LIB = HERE / "_ref" / "libtsref.so"
PORT_LIB = HERE / "_build" / "libtsoracle.so"

INIT_STATE, INIT_GAUSSIAN, INIT_FOURIER = 0, 1, 2


class RefDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int * 3),
        ("prob_lo", C.c_double * 3),
        ("prob_hi", C.c_double * 3),
        ("periodic", C.c_int * 3),
        ("ngrow", C.c_int),
        ("model", C.c_int),
        ("ko_strength", C.c_double),
        ("abl_thickness", C.c_int),
        ("abl_max_strength", C.c_double),
        ("abl_profile", C.c_int),
        ("bc", C.c_int),
        ("bc_values", C.c_double * 12),
        ("dt", C.c_double),
        ("integrator", C.c_int),
        ("block", C.c_int * 3),
        ("c2", C.c_void_p),
    ]


def build() -> None:
    """Builds the oracles in place (make -C oracle)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def from_desc(d, block=(0, 0, 0)) -> RefDesc:
    """RefDesc from any object with the ts_wave_desc field names (e.g. treesap_b200.WaveDesc)."""
    r = RefDesc()
    r.n[:] = list(d.n)
    r.prob_lo[:] = list(d.prob_lo)
    r.prob_hi[:] = list(d.prob_hi)
    r.periodic[:] = list(d.periodic)
    r.ngrow = d.ngrow
    r.model = d.model
    r.ko_strength = d.ko_strength
    r.abl_thickness = d.abl_thickness
    r.abl_max_strength = d.abl_max_strength
    r.abl_profile = d.abl_profile
    r.bc = d.bc
    r.bc_values[:] = list(d.bc_values)
    r.dt = d.dt
    r.integrator = getattr(d, "scheme", getattr(d, "integrator", 1))
    r.block[:] = list(block)
    r.c2 = None
    return r


class Oracle:
    def __init__(self, which: str = "port"):
        path = REF_LIB if which == "ref" else PORT_LIB
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle)")
        self.which = which
        self.lib = C.CDLL(str(path))
        fn = "tsref_run" if which == "ref" else "tso_run"
        self.fn = getattr(self.lib, fn)
        self.fn.restype = C.c_int
        self.fn.argtypes = [C.POINTER(RefDesc), C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        th = getattr(self.lib, "tsref_threads" if which == "ref" else "tso_threads")
        th.restype = C.c_int
        self.threads = th()

    def run(self, desc, nsteps: int, *, state=None, init_kind=INIT_GAUSSIAN, items=None, c2=None, block=(0, 0, 0)):
        """Returns (final valid state [comp][z][y][x], seconds of the step loop, simulation time)."""
        r = from_desc(desc, block) if not isinstance(desc, RefDesc) else desc
        ncomp = 12 if r.model == 1 else 2
        out = np.zeros((ncomp, r.n[2], r.n[1], r.n[0]))
        keep = []
        if c2 is not None:
            c2a = np.ascontiguousarray(c2, dtype=np.float64)
            keep.append(c2a)
            r.c2 = c2a.ctypes.data
        st = None
        if state is not None:
            sa = np.ascontiguousarray(state, dtype=np.float64)
            keep.append(sa)
            st = sa.ctypes.data
            init_kind = INIT_STATE
        it, nit = None, 0
        if items is not None:
            ia = np.ascontiguousarray(items, dtype=np.float64).reshape(-1, 6)
            keep.append(ia)
            it, nit = ia.ctypes.data, len(ia)
        secs, t = C.c_double(), C.c_double()
        rc = self.fn(C.byref(r), init_kind, nit, it, st, nsteps, out.ctypes.data, C.byref(secs), C.byref(t))
        if rc != 0:
            raise RuntimeError(f"oracle {self.which} returned {rc}")
        return out, secs.value, t.value


def available(which: str) -> bool:
    return (REF_LIB if which == "ref" else PORT_LIB).exists()


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def host_cores() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


EXAMPLES_REF_LIB = HERE / "_ref" / "libtsref_examples.so"
EXAMPLES_GPU_LIB = HERE / "_ref" / "libtsb_examples.so"
EXAMPLE_NCOMP = {1: 4, 2: 2, 3: 2}


class ExampleRunner:
    """The reference's example models (and the test-only DerivativeProbeRHS) on either side of
    the example parity tests: `side="ref"` runs the reference integrators on the host
    (libtsref_examples.so), `side="gpu"` the B200 front end (libtsb_examples.so). Both are
    built by the oracle recipe from the same model sources (tests/cpp/examples_run.hpp)."""

    def __init__(self, side: str):
        path = EXAMPLES_REF_LIB if side == "ref" else EXAMPLES_GPU_LIB
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle with the reference sources present)")
        self.lib = C.CDLL(str(path))
        self.fn = getattr(self.lib, "tsref_example_run" if side == "ref" else "tsb_example_run")
        self.fn.restype = C.c_int
        self.fn.argtypes = [C.c_int, C.POINTER(RefDesc), C.c_double, C.c_void_p, C.c_int, C.c_void_p]

    def run(self, example: int, desc: RefDesc, state: np.ndarray, nsteps: int, param: float = 0.0) -> np.ndarray:
        st = np.ascontiguousarray(state, dtype=np.float64)
        out = np.zeros_like(st)
        rc = self.fn(example, C.byref(desc), param, st.ctypes.data, nsteps, out.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"example run returned {rc}")
        return out


def examples_available(side: str) -> bool:
    return (EXAMPLES_REF_LIB if side == "ref" else EXAMPLES_GPU_LIB).exists()
