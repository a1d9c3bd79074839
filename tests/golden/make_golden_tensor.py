"""Fixtures for the 1D / tensor-product aggregation (reference code run here).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_tensor.py [/path/to/reference]

Writes tensor_ext.npz:
  * for several (n, p, cut fraction) the gamma and E of
    polynomial_preserving_extension (code/cut_spline_sbp.py:156-198) on the
    1D cut interval [h * fraction, 1];
  * for one 3D cut box, assemble_cut_3d (code/cut_3d_sbp.py:89-146): its
    tensor E = Ez (x) Ey (x) Ex and the pulled-back mass H.
Inputs/outputs only; no reference source is copied.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
CASES_1D = [(6, 3, 0.35), (5, 2, 0.9), (8, 4, 0.999), (6, 3, 0.0), (12, 5, 0.97)]
BOX = (5, 3, (0.3, 0.6, 0.9))


def main(ref_root: str) -> None:
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(Path(ref_root) / "code"))
    import cut_3d_sbp as c3
    import cut_spline_sbp as c1

    out = {}
    for k, (n, p, frac) in enumerate(CASES_1D):
        b = c1.make_open_uniform_basis(n_elements=n, degree=p)
        m = c1.assemble_cut_matrices(b, left=b.h * frac)
        agg = c1.polynomial_preserving_extension(b, m, support_threshold=0.05)
        out[f"c{k}_meta"] = np.array([n, p, frac])
        out[f"c{k}_gamma"] = agg.gamma
        out[f"c{k}_E"] = agg.E
        out[f"c{k}_interior"] = agg.interior
    out["count"] = np.array(len(CASES_1D))
    n, p, fr = BOX
    ops = c3.assemble_cut_3d(n_elements=n, degree=p, cut_fractions=fr)
    out["box_meta"] = np.array([n, p, *fr])
    out["box_E"] = ops.E
    out["box_H"] = ops.H
    np.savez_compressed(HERE / "tensor_ext.npz", **out)
    print("written", HERE / "tensor_ext.npz")


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
    from oracle.build_ref import reference_root

    main(str(reference_root(sys.argv[1] if len(sys.argv) > 1 else None)))
