"""Ghost-cell enumeration of the fill kernels, checked on the host (no GPU): the enumeration
decodes a flat ghost index into (i, j, k) with 32-bit arithmetic and must visit every ghost cell
of the grown box exactly once (tests/cpp/ghost_enum_check.cu)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_ghost_enumeration_covers_every_ghost_cell_once(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        pytest.skip("nvcc not available")
    exe = tmp_path / "ghost_enum_check"
    subprocess.run([nvcc, "-std=c++20", "-O2", "--expt-relaxed-constexpr", f"-I{ROOT / 'include'}",
                    f"-I{ROOT / 'treesap_b200/cpp/compat'}", f"-I{ROOT / 'treesap_b200/cpp/treesap'}",
                    str(ROOT / "tests/cpp/ghost_enum_check.cu"), "-o", str(exe)], check=True, capture_output=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
