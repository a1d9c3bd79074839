"""Golden vectors of the reference's periodic-hill fast-diagonalisation.

Builds oracle/_ref/hill_ref from the reference's own headers (recipe
oracle/build_ref.py), runs FastDiagHill::solve (and one hill_fastdiag_step)
on a seeded random field for ne=6, nz=12, p=3, and stores operators, z
symbols, inputs and outputs in hill_fastdiag.npz.

    python tests/golden/make_golden_hill.py [/path/to/reference]
"""

from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))


def main(ref_root=None, ne=6, nz=12, seed=99, steps=1):
    from oracle.build_ref import build

    exe = build(ref_root)
    with tempfile.TemporaryDirectory() as td:
        out = Path(td) / "h.bin"
        subprocess.run([str(exe), str(ne), str(nz), str(seed), str(out), str(steps)], check=True)
        raw = np.fromfile(out, dtype=np.float64)
    nr, nz_, a, st = int(raw[0]), int(raw[1]), raw[2], int(raw[3])
    k = 4
    def take(n):
        nonlocal k
        v = raw[k : k + n]
        k += n
        return v
    d = {"nr": nr, "nz": nz_, "a": a, "ne": ne, "seed": seed}
    for name in ("M2", "Qx2", "Qy2", "KN2"):
        d[name] = take(nr * nr).reshape(nr, nr)
    zr = take(3 * nz_)
    d["Mz_row"], d["Sz_row"], d["Kz_row"] = zr[:nz_], zr[nz_ : 2 * nz_], zr[2 * nz_ :]
    for name in ("mu", "sig", "kap"):
        d[name] = take(nz_)
    for name in ("ux", "uy", "uz", "ox", "oy", "oz"):
        d[name] = take(nr * nz_).reshape(nr, nz_)
    if st:
        for name in ("sx", "sy", "sz"):
            d[name] = take(nr * nz_).reshape(nr, nz_)
        d["step_dt"], d["step_fx"] = 0.02, 0.7
    assert k == raw.size
    np.savez_compressed(HERE / "hill_fastdiag.npz", **d)
    print("nr", nr, "nz", nz_, "->", HERE / "hill_fastdiag.npz")


if __name__ == "__main__":
    main(*(sys.argv[1:2] or []))
