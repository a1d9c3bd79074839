"""Recipe: compile the reference's own C++ hill fast-diagonalisation into
oracle/_ref/hill_ref (test infrastructure; outputs only under oracle/_ref/).

The reference path is header-only C++17 (cpp/include/{core,cut,...}), so it
is compiled directly from its sources where they lie -- no reference build
system is run.  Needs the reference tree: an explicit argument, else the
environment variable CUTCELL_REFERENCE_ROOT, else the checkout location this
recipe was written for (READ_ONLY_CHECKOUT).  Every script that reads the
reference resolves its location through ``reference_root``.
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
READ_ONLY_CHECKOUT = "/root/reference"


def reference_root(arg: str | None = None) -> Path:
    """Location of the reference tree (argument > CUTCELL_REFERENCE_ROOT > checkout)."""
    return Path(arg or os.environ.get("CUTCELL_REFERENCE_ROOT") or READ_ONLY_CHECKOUT)


def build(ref_root: str | None = None) -> Path | None:
    inc = reference_root(ref_root) / "cpp" / "include"
    if not inc.exists():
        return None
    out = HERE / "_ref" / "hill_ref"
    out.parent.mkdir(exist_ok=True)
    src = HERE / "hill_ref_main.cpp"
    if out.exists() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    cmd = ["g++", "-std=c++17", "-O2", *[f"-I{inc / d}" for d in ("core", "operators", "solvers", "cut", "io")], str(src), "-o", str(out)]
    subprocess.run(cmd, check=True)
    return out


def build_gpu_run(ref_root: str | None = None) -> Path | None:
    """The reference's own device hill step (cpp/gpu/gpu_run.cu: its kernels
    plus cuBLAS, the baseline GPU time of hill_fastdiag_step), compiled from
    that one source file with nvcc for sm_100a into oracle/_ref/gpu_run."""
    import shutil

    root = reference_root(ref_root)
    src = root / "cpp" / "gpu" / "gpu_run.cu"
    inc = root / "cpp" / "include"
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not src.exists() or not Path(nvcc).exists():
        return None
    out = HERE / "_ref" / "gpu_run"
    out.parent.mkdir(exist_ok=True)
    if out.exists() and out.stat().st_mtime >= src.stat().st_mtime:
        return out
    cmd = [nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           *[f"-I{inc / d}" for d in ("core", "operators", "solvers", "cut", "io")], str(src), "-lcublas", "-o", str(out)]
    subprocess.run(cmd, check=True, capture_output=True)
    return out


if __name__ == "__main__":
    print(build(*sys.argv[1:]))
    print(build_gpu_run(*sys.argv[1:]))
