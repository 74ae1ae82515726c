"""The AMReX plotfile writer of the exporter (util/PlotExporter.hpp), checked on the host: a
plotfile of a known field, written by a small g++ program, read back with tests/plotfile.py."""
import subprocess
from pathlib import Path

import numpy as np

from plotfile import read_plotfile

ROOT = Path(__file__).resolve().parents[1]
INC = ["-I", str(ROOT / "include"), "-I", str(ROOT / "treesap_b200/cpp/compat"), "-I",
       str(ROOT / "treesap_b200/cpp/treesap")]


def test_plotfile_layout_and_data(tmp_path):
    exe = tmp_path / "probe"
    subprocess.run(["g++", "-std=c++20", "-O1", *INC, str(ROOT / "tests/cpp/plotfile_probe.cpp"), "-o", str(exe)],
                   check=True)
    out = tmp_path / "plt00042"
    subprocess.run([str(exe), str(out)], check=True)
    p = read_plotfile(out)
    assert p["names"] == ["phi", "pi", "speed"]
    assert p["dim"] == 3 and p["finest_level"] == 0 and p["coord"] == 0 and p["bwidth"] == 0
    assert p["time"] == 0.125 and p["step"] == 42 and p["level_step"] == 42
    assert p["n"] == [7, 5, 4]
    assert p["prob_lo"] == [-1.0, 0.0, 0.5] and p["prob_hi"] == [1.0, 2.0, 1.5]
    assert np.allclose(p["dx"], [2 / 7, 2 / 5, 1 / 4], rtol=1e-15)
    assert p["grid_phys"] == [[-1.0, 1.0], [0.0, 2.0], [0.5, 1.5]]
    c, k, j, i = np.meshgrid(np.arange(3), np.arange(4), np.arange(5), np.arange(7), indexing="ij")
    want = 1000.0 * c + 100.0 * k + 10.0 * j + i + 0.25
    assert np.array_equal(p["data"], want)
    assert p["min"] == [want[q].min() for q in range(3)]
    assert p["max"] == [want[q].max() for q in range(3)]
