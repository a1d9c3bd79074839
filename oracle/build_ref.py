"""Recipe: compile the reference's own C++ hill fast-diagonalisation into
oracle/_ref/hill_ref (test infrastructure; outputs only under oracle/_ref/).

The reference path is header-only C++17 (cpp/include/{core,cut,...}), so it
is compiled directly from its sources where they lie -- no reference build
system is run.  Needs the reference tree (default /root/reference).
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent


def build(ref_root: str = "/root/reference") -> Path | None:
    inc = Path(ref_root) / "cpp" / "include"
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
