"""Build recipe of the B200 library: nvcc for sm_100a, in-tree.

    python -m treesap_b200.build [--jobs N] [--force]

Compiles every translation unit of treesap_b200/csrc/ into _build/ (in parallel) and links
treesap_b200/libtreesap_b200.so. Objects are rebuilt when their source or any header under
treesap_b200/cpp/, treesap_b200/csrc/ or include/ is newer.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = ROOT / "_build" / "treesap_b200"
LIB = PKG / "libtreesap_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = [
    f"-I{ROOT / 'include'}",
    f"-I{PKG / 'cpp' / 'compat'}",
    f"-I{PKG / 'cpp' / 'treesap'}",
    f"-I{PKG / 'cpp' / 'rhs'}",
]
NVCC_FLAGS = [
    "-std=c++20",
    "-O3",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "--extended-lambda",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "-diag-suppress=20012,20208",
] + ARCH + INCLUDES


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    hs: list[Path] = []
    for d in (PKG / "cpp", CSRC, ROOT / "include"):
        hs += [p for p in d.rglob("*") if p.suffix in (".h", ".hpp", ".cuh", ".H")]
    return hs


def _stale(src: Path, obj: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def compile_one(src: Path, obj: Path, extra: list[str]) -> tuple[Path, float, str]:
    import time

    t0 = time.time()
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    return src, time.time() - t0, r.stderr


def build(jobs: int | None = None, force: bool = False, extra: list[str] | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    extra = extra or []
    srcs = sorted(CSRC.glob("*.cu"))
    newest = max((p.stat().st_mtime for p in _headers()), default=0.0)
    todo = [(s, BUILD / (s.stem + ".o")) for s in srcs if force or _stale(s, BUILD / (s.stem + ".o"), newest)]
    if todo:
        jobs = jobs or min(len(todo), os.cpu_count() or 4)
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for src, secs, err in ex.map(lambda a: compile_one(*a, extra), todo):
                if verbose:
                    print(f"  {src.name}: {secs:.1f}s", file=sys.stderr)
                    if err.strip():
                        print(err, file=sys.stderr)
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    if todo or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true", help="print registers / spills per kernel")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else []
    lib = build(a.jobs, a.force or a.ptxas_verbose, extra, verbose=True)
    print(lib)


if __name__ == "__main__":
    main()
