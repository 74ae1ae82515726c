"""A C++ program written against the header front end (like the reference's example drivers)
runs on the GPU and exports AMReX plotfiles through configureExporter; the exported states
must equal the same model stepped through the C ABI."""
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from plotfile import read_plotfile
from treesap_b200 import TS_BC_DIRICHLET, Integrator
from treesap_b200.configs import wave_desc

pytestmark = pytest.mark.gpu
ROOT = Path(__file__).resolve().parents[1]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = tmp_path_factory.mktemp("drv") / "plotfile_driver"
    inc = [f"-I{ROOT / 'include'}", f"-I{ROOT / 'treesap_b200/cpp/compat'}", f"-I{ROOT / 'treesap_b200/cpp/treesap'}",
           f"-I{ROOT / 'treesap_b200/cpp/rhs'}"]
    cmd = [nvcc, "-std=c++20", "-O3", "--expt-relaxed-constexpr", "--extended-lambda", "-gencode",
           "arch=compute_100a,code=sm_100a", *inc, str(ROOT / "tests/cpp/plotfile_driver.cu"),
           f"-L{ROOT / 'treesap_b200'}", "-ltreesap_b200", "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_front_end_program_exports_plotfiles(driver, ctx, tmp_path):
    env = dict(os.environ, LD_LIBRARY_PATH=f"{ROOT / 'treesap_b200'}:" + os.environ.get("LD_LIBRARY_PATH", ""))
    r = subprocess.run([str(driver), str(tmp_path / "plt")], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Integrator::step() [STEP]" in r.stdout  # the ScopedTimer overview
    d = wave_desc((24, 20, 16), 2, periodic=(0, 0, 0), bc=TS_BC_DIRICHLET, dt=0.25 / 24)
    it = Integrator(ctx, d)
    it.initialise_expressions(["exp(-((x-0.5)^2 + (y-0.5)^2 + (z-0.5)^2)/0.15^2)", "0.0"])
    done = 0
    for step in (0, 2, 4):
        it.step(step - done)
        done = step
        want = it.get_state()
        p = read_plotfile(tmp_path / f"plt{step:05d}")
        assert p["names"] == ["phi", "pi"] and p["step"] == step and p["n"] == [24, 20, 16]
        assert p["time"] == pytest.approx(step * 0.25 / 24, rel=1e-15)
        assert np.array_equal(p["data"], want)
        assert p["max"] == [want[0].max(), want[1].max()]
