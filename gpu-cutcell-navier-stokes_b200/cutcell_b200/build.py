"""Build recipe for libcutcell_b200.so (in-tree, sm_100a).

    python -m cutcell_b200.build          # from gpu-cutcell-navier-stokes_b200/

nvcc cross-compiles without a GPU; the .so lands next to this file so it
travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = ROOT / "csrc"
SOURCES = ["cutcell.cu", "noalloc.cu", "batch.cu", "hilladv.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def build_setup(force: bool = False) -> Path:
    """Host setup library (g++ -O3 -fopenmp), no CUDA."""
    out = PKG / "libcutcell_setup.so"
    src = CSRC / "cutcell_setup.cpp"
    hdr = ROOT.parent / "include" / "cutcell_setup.h"
    if out.exists() and not force and all(out.stat().st_mtime >= d.stat().st_mtime for d in (src, hdr)):
        return out
    # $CXX first; a toolchain without libgomp (OpenMP) falls through to the next
    cands = [c for c in (os.environ.get("CXX"), shutil.which("g++"), "/usr/bin/g++") if c]
    last = None
    for cxx in dict.fromkeys(cands):
        cmd = [cxx, "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", str(src), "-o",
               str(out) + ".tmp"]
        r = subprocess.run(cmd, cwd=str(ROOT), capture_output=True, text=True)
        if r.returncode == 0:
            os.replace(str(out) + ".tmp", out)
            return out
        last = f"{' '.join(cmd)}\n{r.stderr}"
    raise RuntimeError(f"cannot build the setup library:\n{last}")


def build(verbose: bool = False, force: bool = False) -> Path:
    build_setup(force=force)
    out = PKG / "libcutcell_b200.so"
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [ROOT.parent / "include" / "cutcell_b200.h"]
    if out.exists() and not force and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps if d.exists()):
        return out
    cmd = [
        nvcc(),
        *ARCH,
        "-lineinfo",
        "-O3",
        "-std=c++17",
        "-Xcompiler",
        "-fPIC",
        "-shared",
        *(["-Xptxas", "-v"] if verbose else []),
        *[str(CSRC / s) for s in SOURCES],
        "-o",
        str(out) + ".tmp",
    ]
    subprocess.run(cmd, check=True, cwd=str(ROOT))
    os.replace(str(out) + ".tmp", out)
    return out


if __name__ == "__main__":
    p = build(verbose="-v" in sys.argv, force="--force" in sys.argv)
    print(p)
