"""The C ABI library loads, exports every entry point declared in include/treesap_b200.h and
answers the device-independent calls without a GPU (no compute)."""
import ctypes as C
import re
from pathlib import Path

import pytest

import treesap_b200 as tsb

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    txt = (ROOT / "include" / "treesap_b200.h").read_text()
    return sorted(set(re.findall(r"TS_API[^;(]*?\b(ts_\w+)\s*\(", txt)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    assert "ts_integrator_create" in syms and "ts_context_create" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol():
    lib = tsb.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_build_targets_sm100a_only():
    from treesap_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_status_strings_and_version():
    lib = tsb.lib()
    assert lib.ts_abi_version() == 2
    assert lib.ts_status_string(0) == b"TS_OK"
    assert lib.ts_status_string(6) == b"TS_ERR_NO_DEVICE"


@pytest.mark.parametrize("dtype,esize", [(0, 8), (1, 4)])
@pytest.mark.parametrize("ngrow", [1, 2, 3, 4])
def test_field_layout_rules(dtype, esize, ngrow):
    lib = tsb.lib()
    n = (C.c_int * 3)(37, 29, 41)
    L = tsb.FieldLayout()
    assert lib.ts_field_layout_make(n, ngrow, 2, dtype, C.byref(L)) == 0
    a = 32 // esize
    assert L.xoff == -(-ngrow // a) * a  # ngrow rounded up to a 32-byte sector
    assert (L.xoff * esize) % 32 == 0 and (L.px * esize) % 32 == 0  # whole sectors; TMA needs 16 bytes
    assert L.px >= L.xoff + 37 + ngrow and L.py == 29 + 2 * ngrow and L.pz == 41 + 2 * ngrow
    assert lib.ts_field_bytes(C.byref(L)) == L.px * L.py * L.pz * 2 * esize


def test_invalid_arguments_are_rejected():
    lib = tsb.lib()
    L = tsb.FieldLayout()
    assert lib.ts_field_layout_make((C.c_int * 3)(3, 3, 3), 4, 2, 0, C.byref(L)) == 1  # n < ngrow
    assert lib.ts_field_layout_make((C.c_int * 3)(8, 8, 8), 2, 0, 0, C.byref(L)) == 1  # ncomp 0
    # the stage kernels count the rows of a component (y x z with ghosts) in 32 bits
    assert lib.ts_field_layout_make((C.c_int * 3)(64, 46340, 46340), 2, 1, 0, C.byref(L)) == 1
    assert lib.ts_field_layout_make((C.c_int * 3)(64, 46000, 46000), 2, 1, 0, C.byref(L)) == 0
    assert lib.ts_integrator_create(None, None, None) == 1
    assert lib.ts_context_sync(None) == 1


def test_context_without_gpu_reports_no_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert tsb.lib().ts_context_create(0, C.byref(h)) == 6  # TS_ERR_NO_DEVICE, no crash
