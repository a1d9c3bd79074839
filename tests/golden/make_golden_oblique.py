"""Generate the 2D oblique-cut fixtures by running the REFERENCE's own Python
code (imported from its source tree, read-only).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_oblique.py [/path/to/reference]

Writes:
  oblique2d.npz      for a few (n, p, angle, offset) cuts: the full-space forms
                     H, K, Qx, Sx of assemble_oblique_cut_matrices
                     (code/oblique_cut_sbp.py:271-433), gamma and E of
                     polynomial_preserving_oblique_extension (:614-672), the
                     reduced SPD systems 0.5(A + A^T) for A = E^T H E (mass) and
                     E^T (K + H) E (stiffness), and the reference solve_cpu_cg
                     (code/fast_solver_backends.py:90-132) on N(0,1) right-hand
                     sides: iterations, residual and solution;
  oblique_sweep.npz  the 72 committed rows of the reference's oblique sweep
                     (code/results/s6_oblique_sweep_summary.json): p, angle,
                     offset fraction, n, reduced size and cond(sym E^T H E).
Inputs/outputs only; no reference source is copied.
"""

from __future__ import annotations

import json
import os
import sys
from math import pi
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent

CASES = [  # n, p, angle (deg), offset / h
    (6, 3, 12.0, 0.30),
    (8, 5, 37.0, 0.80),
    (6, 4, 44.0, 0.05),
    (12, 3, 3.0, 0.97),
]


def main(ref_root: str) -> None:
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(Path(ref_root) / "code"))
    import cut_spline_sbp as c1
    import fast_solver_backends as fsb
    import oblique_cut_sbp as ob

    out = {}
    for k, (n, p, ang, frac) in enumerate(CASES):
        bx = c1.make_open_uniform_basis(n_elements=n, degree=p)
        by = c1.make_open_uniform_basis(n_elements=n, degree=p)
        cut = ob.HalfPlaneCut.from_angle(ang * pi / 180.0, frac * bx.h)
        m = ob.assemble_oblique_cut_matrices(bx, by, cut)
        agg = ob.polynomial_preserving_oblique_extension(bx, by, m, preserve_degree=p)
        red = ob.pullback_oblique_2d(m, agg.E)
        for name in ("H", "K", "Qx", "Sx"):
            out[f"c{k}_{name}"] = getattr(m, name)
        out[f"c{k}_gamma"] = agg.gamma
        out[f"c{k}_E"] = agg.E
        out[f"c{k}_interior"] = agg.interior
        out[f"c{k}_small"] = agg.small_support
        out[f"c{k}_meta"] = np.array([n, p, ang, frac, agg.polynomial_degree, agg.polynomial_residual])
        for form, M in (("mass", red.H), ("stiffness", red.K + red.H)):
            A = sp.csr_matrix(0.5 * (M + M.T))
            A.sort_indices()
            rng = np.random.default_rng(4321 + 7 * k + (form == "mass"))
            b = rng.standard_normal(A.shape[0])
            x, rep = fsb.solve_cpu_cg(A, b, tol=1e-9, maxiter=20000, preconditioner="jacobi")
            pre = f"c{k}_{form}"
            out[f"{pre}_indptr"] = A.indptr
            out[f"{pre}_indices"] = A.indices
            out[f"{pre}_data"] = A.data
            out[f"{pre}_b"] = b
            out[f"{pre}_x"] = x
            out[f"{pre}_rep"] = np.array([rep.iterations, rep.relative_residual, float(rep.success)])
    out["count"] = np.array(len(CASES))
    np.savez_compressed(HERE / "oblique2d.npz", **out)

    s = json.load(open(Path(ref_root) / "code" / "results" / "s6_oblique_sweep_summary.json"))
    rows = s["rows"]
    cols = ["p", "angle_deg", "offset_fraction", "n_elements", "n_physical_scalar", "cond_H_phys"]
    np.savez_compressed(HERE / "oblique_sweep.npz", columns=np.array(cols),
                        rows=np.array([[float(r[c]) for c in cols] for r in rows]))
    print("oblique fixtures written to", HERE)


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
    from oracle.build_ref import reference_root

    main(str(reference_root(sys.argv[1] if len(sys.argv) > 1 else None)))
