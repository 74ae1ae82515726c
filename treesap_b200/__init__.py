"""ctypes bindings of the treesap-b200 C ABI (include/treesap_b200.h).

The product is the C++20 header front end plus the CUDA library libtreesap_b200.so; this
module is the thin Python binding that tests and bench.py drive it through. There is no
CPU fallback: every call goes to the sm_100a kernels of the library, and loading fails
loudly when the library has not been built.
"""
from __future__ import annotations

import atexit
import ctypes as C
import weakref
from pathlib import Path

import numpy as np

__all__ = [
    "LIB_PATH",
    "TSError",
    "WaveDesc",
    "FieldLayout",
    "lib",
    "Context",
    "Integrator",
    "Batch",
    "Adjoint",
    "TS_EULER",
    "TS_RK4",
    "TS_DOPRI5",
    "TS_F64",
    "TS_F32_STAGE",
    "TS_BC_NOOP",
    "TS_BC_DIRICHLET",
    "TS_INIT_GAUSSIAN",
    "TS_INIT_FOURIER",
    "TS_MODEL_WAVE",
    "TS_MODEL_TENSOR_WAVE",
    "TS_FAULT_NONE",
    "TS_FAULT_SKIP_COPY",
    "TS_FAULT_ALLOC",
]

LIB_PATH = Path(__file__).resolve().with_name("libtreesap_b200.so")

TS_OK = 0
TS_EULER, TS_RK4, TS_DOPRI5 = 0, 1, 2
TS_F64, TS_F32_STAGE = 0, 1
TS_BC_NOOP, TS_BC_DIRICHLET = 0, 1
TS_INIT_STATE, TS_INIT_GAUSSIAN, TS_INIT_FOURIER, TS_INIT_EXPRESSION = 0, 1, 2, 3
TS_MODEL_WAVE, TS_MODEL_TENSOR_WAVE = 0, 1
STATUS_NAMES = {
    0: "TS_OK",
    1: "TS_ERR_INVALID_ARGUMENT",
    2: "TS_ERR_UNSUPPORTED",
    3: "TS_ERR_CUDA",
    4: "TS_ERR_OUT_OF_MEMORY",
    5: "TS_ERR_DEVICE",
    6: "TS_ERR_NO_DEVICE",
    7: "TS_ERR_NONFINITE",
}
TS_FAULT_NONE, TS_FAULT_SKIP_COPY, TS_FAULT_ALLOC = 0, 1, 2


class TSError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        super().__init__(f"{what}: {STATUS_NAMES.get(status, status)}" + (f" ({detail})" if detail else ""))


class WaveDesc(C.Structure):
    """Mirror of ts_wave_desc."""

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
        ("scheme", C.c_int),
        ("precision", C.c_int),
        ("c2", C.c_void_p),
        ("block", C.c_int * 3),
        ("rtol", C.c_double),
        ("atol", C.c_double),
    ]

    def ncomp(self) -> int:
        return 12 if self.model == TS_MODEL_TENSOR_WAVE else 2

    def shape(self) -> tuple[int, int, int, int]:
        """Valid-state array shape (comp, z, y, x)."""
        return (self.ncomp(), self.n[2], self.n[1], self.n[0])


class FieldLayout(C.Structure):
    """Mirror of ts_field_layout."""

    _fields_ = [
        ("n", C.c_int * 3),
        ("ngrow", C.c_int),
        ("ncomp", C.c_int),
        ("dtype", C.c_int),
        ("xoff", C.c_int),
        ("reserved", C.c_int),
        ("px", C.c_longlong),
        ("py", C.c_longlong),
        ("pz", C.c_longlong),
    ]


_lib = None


def lib() -> C.CDLL:
    """The loaded C-ABI library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m treesap_b200.build`")
    L = C.CDLL(str(LIB_PATH))
    vp, i, d, ll = C.c_void_p, C.c_int, C.c_double, C.c_longlong
    sig = {
        "ts_abi_version": (i, []),
        "ts_status_string": (C.c_char_p, [i]),
        "ts_context_create": (i, [i, C.POINTER(vp)]),
        "ts_context_destroy": (i, [vp]),
        "ts_context_sync": (i, [vp]),
        "ts_context_last_error": (C.c_char_p, [vp]),
        "ts_context_stream": (vp, [vp]),
        "ts_context_error_word": (vp, [vp]),
        "ts_context_sm_count": (i, [vp]),
        "ts_context_inject_fault": (i, [vp, i, ll]),
        "ts_context_take_stage_fault": (i, [vp, C.POINTER(i), C.POINTER(C.c_ulonglong)]),
        "ts_field_layout_make": (i, [C.POINTER(i), i, i, i, C.POINTER(FieldLayout)]),
        "ts_field_bytes": (ll, [C.POINTER(FieldLayout)]),
        "ts_field_tensor_map": (i, [C.POINTER(FieldLayout), vp, i, i, vp]),
        "ts_integrator_create": (i, [vp, C.POINTER(WaveDesc), C.POINTER(vp)]),
        "ts_integrator_destroy": (i, [vp]),
        "ts_integrator_ncomp": (i, [vp]),
        "ts_integrator_initialise": (i, [vp, i, i, vp]),
        "ts_integrator_set_state": (i, [vp, vp, i]),
        "ts_integrator_get_state": (i, [vp, vp, i]),
        "ts_integrator_step": (i, [vp, i]),
        "ts_integrator_run": (i, [vp, vp, i, vp]),
        "ts_integrator_time": (i, [vp, C.POINTER(d), C.POINTER(ll)]),
        "ts_integrator_state_field": (i, [vp, C.POINTER(vp), C.POINTER(FieldLayout)]),
        "ts_integrator_use_graph": (i, [vp, i]),
        "ts_integrator_check_finite": (i, [vp]),
        "ts_integrator_adaptive_stats": (i, [vp, C.POINTER(ll), C.POINTER(ll), C.POINTER(d), C.POINTER(d)]),
        "ts_integrator_create_slab": (i, [vp, C.POINTER(WaveDesc), i, i, i, i, C.POINTER(vp)]),
        "ts_slab_stages": (i, [vp]),
        "ts_slab_prepare": (i, [vp, i]),
        "ts_slab_send_planes": (i, [vp, i, i, C.POINTER(vp), C.POINTER(ll), C.POINTER(ll), C.POINTER(i)]),
        "ts_slab_receive_planes": (i, [vp, i, i, vp]),
        "ts_slab_fill": (i, [vp, i]),
        "ts_slab_launch": (i, [vp, i]),
        "ts_slab_finish": (i, [vp]),
        "ts_integrator_last_step_timing": (i, [vp, C.POINTER(d), C.POINTER(ll)]),
        "ts_integrator_profile": (i, [vp, i, i, C.POINTER(ll), C.POINTER(d)]),
        "ts_integrator_set_launch_shape": (i, [vp, i, i]),
        "ts_integrator_initialise_expressions": (i, [vp, i, vp]),
        "ts_expression_eval": (i, [C.c_char_p, i, vp, vp, vp, vp]),
        "ts_batch_create": (i, [vp, vp, i, C.POINTER(vp)]),
        "ts_batch_destroy": (i, [vp]),
        "ts_batch_size": (i, [vp]),
        "ts_batch_initialise": (i, [vp, i, i, i, vp]),
        "ts_batch_set_state": (i, [vp, i, vp, i]),
        "ts_batch_get_state": (i, [vp, i, vp, i]),
        "ts_batch_step": (i, [vp, i]),
        "ts_batch_use_graph": (i, [vp, i]),
        "ts_batch_set_launch_shape": (i, [vp, i, i]),
        "ts_batch_autotune": (i, [vp, i, C.POINTER(i), C.POINTER(i)]),
        "ts_batch_last_step_timing": (i, [vp, C.POINTER(d), C.POINTER(ll)]),
        "ts_adjoint_create": (i, [vp, C.POINTER(WaveDesc), i, C.POINTER(vp)]),
        "ts_adjoint_destroy": (i, [vp]),
        "ts_adjoint_forward": (i, [vp, vp, vp, vp, i, vp, vp]),
        "ts_adjoint_gradient": (i, [vp, vp, vp, vp, i, vp, C.POINTER(d), vp, vp, vp]),
        "ts_adjoint_tangent": (i, [vp, vp, vp, vp, vp, vp, vp, i, vp, vp]),
        "ts_adjoint_gradient_f32": (i, [vp, vp, vp, vp, i, vp, C.POINTER(d), vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _check(status: int, what: str, ctx: "Context | None" = None) -> None:
    if status != TS_OK:
        detail = ""
        if ctx is not None and ctx.handle:
            detail = (lib().ts_context_last_error(ctx.handle) or b"").decode()
        raise TSError(status, what, detail)


_live_contexts: weakref.WeakSet = weakref.WeakSet()


@atexit.register
def _close_live_contexts() -> None:
    """Closes every context still open when the interpreter exits, each after its integrators,
    batches and adjoints, while the interpreter and the library are still intact (module
    teardown would otherwise destroy handles in no defined order)."""
    for ctx in list(_live_contexts):
        try:
            ctx.close()
        except Exception:
            pass


class Context:
    """One device, one CUDA stream (ts_context)."""

    def __init__(self, device: int = 0):
        self.handle = C.c_void_p()
        self._dependents = weakref.WeakSet()  # integrators / batches, destroyed before the context
        _check(lib().ts_context_create(device, C.byref(self.handle)), "ts_context_create")
        _live_contexts.add(self)

    def _adopt(self, obj) -> None:
        self._dependents.add(obj)

    def sync(self) -> None:
        _check(lib().ts_context_sync(self.handle), "ts_context_sync", self)

    def inject_fault(self, fault: int, arg: int = 0) -> None:
        """Test hook (ts_context_inject_fault): TS_FAULT_SKIP_COPY / TS_FAULT_ALLOC / TS_FAULT_NONE."""
        _check(lib().ts_context_inject_fault(self.handle, fault, arg), "ts_context_inject_fault", self)

    @property
    def stream(self) -> int:
        return lib().ts_context_stream(self.handle) or 0

    @property
    def sm_count(self) -> int:
        return lib().ts_context_sm_count(self.handle)

    def close(self) -> None:
        if self.handle:
            for dep in list(self._dependents):
                dep.close()
            lib().ts_context_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Integrator:
    """A built-in model integrator (ts_integrator)."""

    def __init__(self, ctx: Context, desc: WaveDesc, c2: np.ndarray | None = None):
        self.ctx = ctx
        self.desc = desc
        self._c2 = None
        if c2 is not None:
            self._c2 = np.ascontiguousarray(c2, dtype=np.float64)
            desc.c2 = self._c2.ctypes.data
        self.handle = C.c_void_p()
        _check(lib().ts_integrator_create(ctx.handle, C.byref(desc), C.byref(self.handle)), "ts_integrator_create", ctx)
        ctx._adopt(self)
        self.shape = desc.shape()

    def initialise(self, kind: int, items: np.ndarray) -> None:
        items = np.ascontiguousarray(items, dtype=np.float64).reshape(-1, 6)
        _check(
            lib().ts_integrator_initialise(self.handle, kind, len(items), items.ctypes.data),
            "ts_integrator_initialise",
            self.ctx,
        )

    def initialise_expressions(self, exprs: list[str]) -> None:
        """FunctionInit: one expression of x, y, z per component."""
        arr = (C.c_char_p * len(exprs))(*[e.encode() for e in exprs])
        _check(lib().ts_integrator_initialise_expressions(self.handle, len(exprs), C.cast(arr, C.c_void_p)),
               "ts_integrator_initialise_expressions", self.ctx)

    def set_state(self, state: np.ndarray) -> None:
        a = np.ascontiguousarray(state, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        _check(lib().ts_integrator_set_state(self.handle, a.ctypes.data, 0), "ts_integrator_set_state", self.ctx)
        self.ctx.sync()  # the host buffer may be freed by the caller

    def set_state_device(self, dev_ptr: int) -> None:
        _check(lib().ts_integrator_set_state(self.handle, dev_ptr, 1), "ts_integrator_set_state", self.ctx)

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.shape, dtype=np.float64)
        _check(lib().ts_integrator_get_state(self.handle, out.ctypes.data, 0), "ts_integrator_get_state", self.ctx)
        return out

    def step(self, nsteps: int = 1) -> None:
        _check(lib().ts_integrator_step(self.handle, nsteps), "ts_integrator_step", self.ctx)

    def run(self, host_in: np.ndarray, nsteps: int, host_out: np.ndarray) -> None:
        _check(
            lib().ts_integrator_run(self.handle, host_in.ctypes.data, nsteps, host_out.ctypes.data),
            "ts_integrator_run",
            self.ctx,
        )

    def adaptive_stats(self) -> dict:
        """TS_DOPRI5: accepted / rejected steps, the next proposed dt and the last error norm."""
        a, r, dt, e = C.c_longlong(), C.c_longlong(), C.c_double(), C.c_double()
        _check(lib().ts_integrator_adaptive_stats(self.handle, C.byref(a), C.byref(r), C.byref(dt), C.byref(e)),
               "ts_integrator_adaptive_stats", self.ctx)
        return {"accepted": a.value, "rejected": r.value, "next_dt": dt.value, "last_error": e.value}

    def check_finite(self) -> None:
        """Raises TSError(TS_ERR_NONFINITE) when the state holds NaN or infinite values."""
        _check(lib().ts_integrator_check_finite(self.handle), "ts_integrator_check_finite", self.ctx)

    def use_graph(self, enable: bool = True) -> None:
        _check(lib().ts_integrator_use_graph(self.handle, int(enable)), "ts_integrator_use_graph", self.ctx)

    def time(self) -> tuple[float, int]:
        t, s = C.c_double(), C.c_longlong()
        _check(lib().ts_integrator_time(self.handle, C.byref(t), C.byref(s)), "ts_integrator_time", self.ctx)
        return t.value, s.value

    def last_step_timing(self) -> tuple[float, int]:
        ms, n = C.c_double(), C.c_longlong()
        _check(lib().ts_integrator_last_step_timing(self.handle, C.byref(ms), C.byref(n)), "timing", self.ctx)
        return ms.value, n.value

    def profile(self, nsteps: int, nclasses: int = 5) -> tuple[list[int], list[float]]:
        """Per kernel class (0 ghost fill, 1+s stage s): launches and total device ms over nsteps steps."""
        n = (C.c_longlong * nclasses)()
        ms = (C.c_double * nclasses)()
        _check(lib().ts_integrator_profile(self.handle, nsteps, nclasses, n, ms), "ts_integrator_profile", self.ctx)
        return list(n), list(ms)

    def set_launch_shape(self, rows: int = 0, chunks: int = 0) -> None:
        _check(lib().ts_integrator_set_launch_shape(self.handle, rows, chunks), "set_launch_shape", self.ctx)

    def state_field(self) -> tuple[int, FieldLayout]:
        p, L = C.c_void_p(), FieldLayout()
        _check(lib().ts_integrator_state_field(self.handle, C.byref(p), C.byref(L)), "state_field", self.ctx)
        return p.value or 0, L

    def close(self) -> None:
        if self.handle:
            lib().ts_integrator_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Independent instances of the scalar wave model advanced together (ts_batch)."""

    def __init__(self, ctx: Context, descs: list[WaveDesc]):
        self.ctx = ctx
        self.descs = (WaveDesc * len(descs))(*descs)
        self.shapes = [d.shape() for d in descs]
        self.handle = C.c_void_p()
        _check(lib().ts_batch_create(ctx.handle, C.cast(self.descs, C.c_void_p), len(descs), C.byref(self.handle)),
               "ts_batch_create", ctx)
        ctx._adopt(self)

    def __len__(self) -> int:
        return lib().ts_batch_size(self.handle)

    def initialise(self, instance: int, kind: int, items: np.ndarray) -> None:
        items = np.ascontiguousarray(items, dtype=np.float64).reshape(-1, 6)
        _check(lib().ts_batch_initialise(self.handle, instance, kind, len(items), items.ctypes.data),
               "ts_batch_initialise", self.ctx)

    def set_state(self, instance: int, state: np.ndarray) -> None:
        a = np.ascontiguousarray(state, dtype=np.float64)
        assert a.shape == self.shapes[instance], (a.shape, self.shapes[instance])
        _check(lib().ts_batch_set_state(self.handle, instance, a.ctypes.data, 0), "ts_batch_set_state", self.ctx)
        self.ctx.sync()

    def get_state(self, instance: int) -> np.ndarray:
        out = np.empty(self.shapes[instance], dtype=np.float64)
        _check(lib().ts_batch_get_state(self.handle, instance, out.ctypes.data, 0), "ts_batch_get_state", self.ctx)
        return out

    def step(self, nsteps: int = 1) -> None:
        _check(lib().ts_batch_step(self.handle, nsteps), "ts_batch_step", self.ctx)

    def use_graph(self, enable: bool = True) -> None:
        _check(lib().ts_batch_use_graph(self.handle, int(enable)), "ts_batch_use_graph", self.ctx)

    def set_launch_shape(self, rows: int = 0, zchunk: int = 0) -> None:
        _check(lib().ts_batch_set_launch_shape(self.handle, rows, zchunk), "ts_batch_set_launch_shape", self.ctx)

    def autotune(self, trial_steps: int = 3) -> tuple[int, int]:
        r, z = C.c_int(), C.c_int()
        _check(lib().ts_batch_autotune(self.handle, trial_steps, C.byref(r), C.byref(z)), "ts_batch_autotune",
               self.ctx)
        return r.value, z.value

    def last_step_timing(self) -> tuple[float, int]:
        ms, n = C.c_double(), C.c_longlong()
        _check(lib().ts_batch_last_step_timing(self.handle, C.byref(ms), C.byref(n)), "ts_batch_timing", self.ctx)
        return ms.value, n.value

    def close(self) -> None:
        if self.handle:
            lib().ts_batch_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _ptr(a: np.ndarray | None) -> int | None:
    return None if a is None else a.ctypes.data


class Adjoint:
    """Discrete adjoint and tangent-linear model of the variable-speed wave system (ts_adjoint).

    Arrays are (nz, ny, nx) float64 host arrays of the valid cells; c is the wave speed.
    """

    def __init__(self, ctx: Context, desc: WaveDesc, checkpoint_every: int = 20):
        self.ctx = ctx
        self.shape = (desc.n[2], desc.n[1], desc.n[0])
        self.handle = C.c_void_p()
        _check(lib().ts_adjoint_create(ctx.handle, C.byref(desc), checkpoint_every, C.byref(self.handle)),
               "ts_adjoint_create", ctx)
        ctx._adopt(self)

    def _in(self, a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        return a

    def forward(self, phi0, pi0, c, nsteps: int):
        phi0, pi0, c = self._in(phi0), self._in(pi0), self._in(c)
        phi, pi = np.empty(self.shape), np.empty(self.shape)
        _check(lib().ts_adjoint_forward(self.handle, _ptr(phi0), _ptr(pi0), _ptr(c), nsteps, _ptr(phi), _ptr(pi)),
               "ts_adjoint_forward", self.ctx)
        return phi, pi

    def gradient(self, phi0, pi0, c, nsteps: int, target):
        """(J, dJ/dphi0, dJ/dpi0, dJ/dc) for J = 1/2 sum (phi(T) - target)^2."""
        phi0, pi0, c, target = self._in(phi0), self._in(pi0), self._in(c), self._in(target)
        gphi, gpi, gc = np.empty(self.shape), np.empty(self.shape), np.empty(self.shape)
        loss = C.c_double()
        _check(lib().ts_adjoint_gradient(self.handle, _ptr(phi0), _ptr(pi0), _ptr(c), nsteps, _ptr(target),
                                         C.byref(loss), _ptr(gphi), _ptr(gpi), _ptr(gc)),
               "ts_adjoint_gradient", self.ctx)
        return loss.value, gphi, gpi, gc

    def gradient_f32(self, phi0, pi0, c, nsteps: int, target, speed: bool = True):
        """FP32-stage form: (J, dJ/dphi0, dJ/dpi0, dJ/dc); dJ/dc is None when speed is False
        (the state gradient alone needs no checkpoints)."""
        phi0, pi0, c, target = self._in(phi0), self._in(pi0), self._in(c), self._in(target)
        gphi, gpi = np.empty(self.shape), np.empty(self.shape)
        gc = np.empty(self.shape) if speed else None
        loss = C.c_double()
        _check(lib().ts_adjoint_gradient_f32(self.handle, _ptr(phi0), _ptr(pi0), _ptr(c), nsteps, _ptr(target),
                                             C.byref(loss), _ptr(gphi), _ptr(gpi), _ptr(gc)),
               "ts_adjoint_gradient_f32", self.ctx)
        return loss.value, gphi, gpi, gc

    def tangent(self, phi0, pi0, c, dphi0, dpi0, dc, nsteps: int):
        args = [self._in(a) for a in (phi0, pi0, c, dphi0, dpi0, dc)]
        dphi, dpi = np.empty(self.shape), np.empty(self.shape)
        _check(lib().ts_adjoint_tangent(self.handle, *[_ptr(a) for a in args], nsteps, _ptr(dphi), _ptr(dpi)),
               "ts_adjoint_tangent", self.ctx)
        return dphi, dpi

    def close(self) -> None:
        if self.handle:
            lib().ts_adjoint_destroy(self.handle)
            self.handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def expression_eval(expr: str, x, y, z) -> np.ndarray:
    """Host evaluation of an initial-condition expression (the program the device runs)."""
    x, y, z = (np.ascontiguousarray(np.broadcast_to(a, np.broadcast(x, y, z).shape), dtype=np.float64)
               for a in (x, y, z))
    out = np.empty(x.shape)
    _check(lib().ts_expression_eval(expr.encode(), x.size, x.ctypes.data, y.ctypes.data, z.ctypes.data,
                                    out.ctypes.data), f"ts_expression_eval({expr!r})")
    return out
