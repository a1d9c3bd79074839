"""Fixtures for the tensor cut-box forms and the two Poisson wrappers whose
dense solves route through solve_spd (the reference code run here).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden_tensorbox.py [/path/to/reference]

Writes tensor_forms.npz:
  * for each box (n, p, cut fractions): assemble_cut_3d (code/cut_3d_sbp.py:89-146)
    forms H, K, Qx, Qy, Qz, Sx, Sy, Sz applied to three seeded N(0, 1)
    vectors (F @ V, so the dense N x N forms need not be stored), their
    reduced size, and green_residuals_3d (:149-154);
  * solve_poisson_3d (:386-531) at two sizes: the reduced right-hand side and
    solution its np.linalg.solve (:503) receives and returns, and its
    relative L2 / H1 / L-infinity errors;
  * solve_poisson_circular (code/cut_pde_solve.py:316-446) at two sizes: the
    system matrix (as CSR), right-hand side and solution of its
    np.linalg.solve (:446).
The solves are captured by wrapping np.linalg.solve for the duration of the
call (the system solve is the largest captured one); inputs/outputs only, no
reference source is copied.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
BOXES = [(5, 3, (0.3, 0.6, 0.9)), (4, 2, (0.6, 0.6, 0.6)), (6, 4, (0.95, 0.0, 0.5))]
POISSON_3D = [(4, 3, (0.6, 0.6, 0.6)), (6, 3, (0.6, 0.6, 0.6))]
CIRCULAR = [(3, 8), (2, 12)]


class _Capture:
    def __init__(self):
        self.calls = []
        self._orig = np.linalg.solve

    def __enter__(self):
        orig = self._orig

        def solve(A, b):
            x = orig(A, b)
            self.calls.append((np.array(A, copy=True), np.array(b, copy=True), np.array(x, copy=True)))
            return x

        np.linalg.solve = solve
        return self

    def __exit__(self, *exc):
        np.linalg.solve = self._orig


def main(ref_root: str) -> None:
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(Path(ref_root) / "code"))
    import cut_3d_sbp as c3
    import cut_pde_solve as cp

    out = {}
    for k, (n, p, fr) in enumerate(BOXES):
        ops = c3.assemble_cut_3d(n_elements=n, degree=p, cut_fractions=fr)
        N = ops.H.shape[0]
        V = np.random.default_rng(777 + k).standard_normal((N, 3))
        out[f"b{k}_meta"] = np.array([n, p, *fr])
        for name in ("H", "K", "Qx", "Qy", "Qz", "Sx", "Sy", "Sz"):
            out[f"b{k}_{name}V"] = getattr(ops, name) @ V
        out[f"b{k}_V"] = V
        out[f"b{k}_green"] = np.array(c3.green_residuals_3d(ops))
    out["n_boxes"] = np.array(len(BOXES))
    for k, (n, p, fr) in enumerate(POISSON_3D):
        with _Capture() as cap:
            r = c3.solve_poisson_3d(n_elements=n, degree=p, cut_fractions=fr)
        # the system solve is the largest one (the extension's moment solves are tiny)
        _, b, x = max(cap.calls, key=lambda c: c[0].shape[0])
        out[f"p{k}_meta"] = np.array([n, p, *fr])
        out[f"p{k}_rhs"] = b
        out[f"p{k}_x"] = x
        out[f"p{k}_err"] = np.array([r["relative_l2_error"], r["relative_h1_error"], r["relative_linf_error"]])
    out["n_poisson"] = np.array(len(POISSON_3D))
    for k, (p, n) in enumerate(CIRCULAR):
        with _Capture() as cap:
            cp.solve_poisson_circular(p, n)
        A, b, x = max(cap.calls, key=lambda c: c[0].shape[0])
        As = sp.csr_matrix(A)
        out[f"c{k}_meta"] = np.array([p, n])
        out[f"c{k}_data"], out[f"c{k}_indices"], out[f"c{k}_indptr"] = As.data, As.indices, As.indptr
        out[f"c{k}_rhs"] = b
        out[f"c{k}_x"] = x
    out["n_circular"] = np.array(len(CIRCULAR))
    np.savez_compressed(HERE / "tensor_forms.npz", **out)
    print("written", HERE / "tensor_forms.npz")


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
    from oracle.build_ref import reference_root

    main(str(reference_root(sys.argv[1] if len(sys.argv) > 1 else None)))
