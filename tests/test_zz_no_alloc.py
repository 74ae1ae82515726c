"""ts_wave_rk4_steps_noalloc: the RK4 entry point for callers that may not allocate device memory.

Callers that hand all device memory to their own pool, or that cannot let cudaMalloc /
cudaFree synchronise the device under their other streams, pass a state buffer they already
own; the entry point keeps its RK4 stage registers in a static device array instead of
allocating. This checks, through the C ABI, that two calls in a row on the same buffer give
the same states as the allocating ts_integrator path (FP64 tolerance of the parity tests:
relative max-norm <= 1e-12), and that a domain too large for the static array is refused.
The file sorts last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import treesap_b200 as tsb
from treesap_b200.configs import wave_desc

pytestmark = pytest.mark.gpu
TOL = 1e-12


def noalloc_fn():
    f = tsb.lib().ts_wave_rk4_steps_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(tsb.WaveDesc), C.c_void_p, C.c_int, C.c_void_p]
    return f


def layout_of(desc):
    L = tsb.FieldLayout()
    n = (C.c_int * 3)(*desc.n)
    assert tsb.lib().ts_field_layout_make(n, 2, 2, tsb.TS_F64, C.byref(L)) == 0
    return L


def to_padded(state, L):
    """Valid cells [comp][z][y][x] -> the library's padded field layout (ghost cells zero)."""
    pad = np.zeros((2, L.pz, L.py, L.px))
    g = L.ngrow
    pad[:, g:g + L.n[2], g:g + L.n[1], L.xoff:L.xoff + L.n[0]] = state
    return pad


def from_padded(pad, L):
    g = L.ngrow
    return pad[:, g:g + L.n[2], g:g + L.n[1], L.xoff:L.xoff + L.n[0]]


def relerr(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


def initial_state(rng):
    z, y, x = np.meshgrid(*(np.arange(m) / m for m in (44, 36, 40)), indexing="ij")
    s0 = np.stack([np.sin(2 * np.pi * (x + 2 * z)) * np.exp(-((y - 0.5) / 0.2) ** 2), 0.1 * np.cos(2 * np.pi * y)])
    return s0 + 0.01 * rng.standard_normal(s0.shape)


@pytest.mark.parametrize("bc", [tsb.TS_BC_DIRICHLET, tsb.TS_BC_NOOP])
@pytest.mark.parametrize("ko", [0.0, 0.1])
def test_noalloc_matches_allocating_path_on_two_calls(ctx, bc, ko):
    import torch

    desc = wave_desc((40, 36, 44), 2, periodic=(1, 0, 1), ko=ko, bc=bc, bc_values=(0.2, 0.0), dt=0.2 / 44)
    s0 = initial_state(np.random.default_rng(7))

    ref = tsb.Integrator(ctx, desc)
    ref.set_state(s0)
    ref.step(3)
    ref3 = ref.get_state()
    ref.step(4)
    ref7 = ref.get_state()
    ctx.sync()
    ref.close()

    L = layout_of(desc)
    dev = torch.from_numpy(to_padded(s0, L)).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    f = noalloc_fn()
    assert f(C.byref(desc), dev.data_ptr(), 3, stream) == 0
    got3 = from_padded(dev.cpu().numpy(), L)
    assert relerr(got3, ref3) <= TOL
    assert f(C.byref(desc), dev.data_ptr(), 4, stream) == 0
    got7 = from_padded(dev.cpu().numpy(), L)
    assert relerr(got7, ref7) <= TOL


def test_noalloc_zero_steps_leaves_the_state_unchanged():
    import torch

    desc = wave_desc((40, 36, 44), 2, periodic=(1, 0, 1), ko=0.1, bc=tsb.TS_BC_DIRICHLET, dt=0.2 / 44)
    L = layout_of(desc)
    pad = to_padded(initial_state(np.random.default_rng(11)), L)
    dev = torch.from_numpy(pad).cuda()
    assert noalloc_fn()(C.byref(desc), dev.data_ptr(), 0, None) == 0
    assert np.array_equal(dev.cpu().numpy(), pad)


def test_noalloc_allocates_no_device_memory():
    """After a first call (which looks up the scratch array's address), further calls leave the
    device's free memory unchanged: the stage registers come from the static array."""
    import torch

    desc = wave_desc((40, 36, 44), 2, periodic=(1, 0, 1), ko=0.1, bc=tsb.TS_BC_DIRICHLET, dt=0.2 / 44)
    L = layout_of(desc)
    dev = torch.from_numpy(to_padded(initial_state(np.random.default_rng(5)), L)).cuda()
    f = noalloc_fn()
    assert f(C.byref(desc), dev.data_ptr(), 1, None) == 0
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert f(C.byref(desc), dev.data_ptr(), 2, None) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


def test_noalloc_refuses_domains_beyond_its_scratch():
    import torch

    desc = wave_desc(160, 2, ko=0.1)  # three padded 160^3 fields exceed TS_NOALLOC_SCRATCH_BYTES
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    assert noalloc_fn()(C.byref(desc), buf.data_ptr(), 1, None) == 1  # TS_ERR_INVALID_ARGUMENT
    other = wave_desc(32, 4, ko=0.1)  # outside the supported model set
    assert noalloc_fn()(C.byref(other), buf.data_ptr(), 1, None) == 2  # TS_ERR_UNSUPPORTED
