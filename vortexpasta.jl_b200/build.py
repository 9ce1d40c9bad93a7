"""Build recipe for libvpbs.so (sm_100a) -- invoked by __graft_entry__.build() and the tests.

The library is compiled in-tree with nvcc and linked against the CUDA runtime and cuFFT.
Run as ``python vortexpasta.jl_b200/build.py`` or call ``build_library()``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "lib"
LIB = OUT_DIR / "libvpbs.so"
SOURCES = ["api.cu", "geometry.cu", "shortrange.cu", "longrange.cu", "features.cu", "mlp.cu", "timestep.cu", "diagnostics.cu", "splitting.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_library(force: bool = False, verbose: bool = False, extra_flags=()) -> Path:
    """Compile every CUDA source of the package into lib/libvpbs.so (incremental)."""
    OUT_DIR.mkdir(exist_ok=True)
    obj_dir = OUT_DIR / "obj"
    obj_dir.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    headers = list(CSRC.glob("*.cuh")) + [ROOT / "include" / "vpbs.h"]
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
                    "-I", str(CSRC), "--expt-relaxed-constexpr"] + list(extra_flags)
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = obj_dir / (s.stem + ".o")
        objs.append(o)
        if force or _stale(o, [s, *headers]):
            cmd = [nvcc, *flags, "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcufft", "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True,
                  extra_flags=["-Xptxas", "-v"] if "--ptxas" in sys.argv else ())
