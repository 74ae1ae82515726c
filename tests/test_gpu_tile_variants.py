"""Stage-kernel tile configurations agree bitwise.

The tiling (cells per thread along x, rows per consumer warp, tile height, circular,
shifted or no register queue, prefetch depth) only changes which thread evaluates which cell and
where the operands wait, never the per-cell arithmetic. tests/cpp/tile_variant_driver.cu is
built once per configuration (compile-time switches of the front end) and every build must
write the same bytes for the FP64 and the FP32-stage forms on a ragged 72 x 45 x 37 box
(partial tiles in x, y and z chunks)."""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]

VARIANTS = {
    "default": [],
    "shifted FP64 queue": ["-DTREESAP_B200_QROT_F64=0"],
    "circular FP32 queue": ["-DTREESAP_B200_QROT_F32=1"],
    "two rows per warp": ["-DTREESAP_B200_TILE_F64=2105421", "-DTREESAP_B200_TILE_F32=2105421"],
    "two FP64 cells per thread, short prefetch": ["-DTREESAP_B200_TILE_F64=204221", "-DTREESAP_B200_TILE_F32=103221"],
    "z taps from global memory": ["-DTREESAP_B200_QUEUE_MAX_COMPONENTS=0"],
    # bounds-checked build: every shared-memory and global stencil access is range-checked and an
    # out-of-range index would set the device error word (the test program then exits non-zero)
    "bounds-checked": ["-DTREESAP_B200_CHECK=1"],
    "bounds-checked, z taps from global memory": ["-DTREESAP_B200_CHECK=1", "-DTREESAP_B200_QUEUE_MAX_COMPONENTS=0"],
}


def _build(tmp: Path, name: str, flags: list[str]) -> Path:
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp / name.replace(" ", "_").replace(",", "")
    inc = [f"-I{ROOT / 'include'}", f"-I{ROOT / 'treesap_b200/cpp/compat'}", f"-I{ROOT / 'treesap_b200/cpp/treesap'}",
           f"-I{ROOT / 'treesap_b200/cpp/rhs'}"]
    cmd = [nvcc, "-std=c++20", "-O3", "--expt-relaxed-constexpr", "--extended-lambda", "-diag-suppress=20011,20014",
           "-gencode", "arch=compute_100a,code=sm_100a", *inc, *flags, str(ROOT / "tests/cpp/tile_variant_driver.cu"),
           f"-L{ROOT / 'treesap_b200'}", "-ltreesap_b200", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


@pytest.fixture(scope="module")
def outputs(tmp_path_factory):
    tmp = tmp_path_factory.mktemp("tiles")
    env = dict(os.environ, LD_LIBRARY_PATH=f"{ROOT / 'treesap_b200'}:" + os.environ.get("LD_LIBRARY_PATH", ""))
    res = {}
    for name, flags in VARIANTS.items():
        exe = _build(tmp, name, flags)
        out = tmp / (exe.name + ".bin")
        r = subprocess.run([str(exe), str(out)], env=env, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (name, r.stderr[-2000:])
        res[name] = np.fromfile(out, dtype=np.float64).reshape(2, 2, 37, 45, 72)
    return res


@pytest.mark.parametrize("name", [v for v in VARIANTS if v != "default"])
def test_tile_configuration_is_bitwise_neutral(outputs, name):
    ref, got = outputs["default"], outputs[name]
    assert np.isfinite(ref).all() and np.abs(ref).max() > 0.1
    for form in range(2):
        assert np.array_equal(got[form], ref[form]), (name, form, np.abs(got[form] - ref[form]).max())


def test_fp32_stage_form_tracks_fp64(outputs):
    ref = outputs["default"]
    assert np.abs(ref[1] - ref[0]).max() <= 1e-6 * np.abs(ref[0]).max()
