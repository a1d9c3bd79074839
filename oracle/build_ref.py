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


if __name__ == "__main__":
    print(build(*sys.argv[1:]))
