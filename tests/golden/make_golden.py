"""Generate the golden fixtures in this folder by running the REFERENCE's own
Python code (imported from its source tree, read-only).

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py [/path/to/reference]

Writes:
  cut1d.npz        1D cut-interval forms of assemble_cut_matrices
                   (code/cut_spline_sbp.py:90-129) for a few cut positions;
  ext3d_bell.npz   gamma and E of polynomial_preserving_extension_3d
                   (code/bell_3d_core.py:471-542) on the 3D bell at n=20, p=2
                   (the benchmark system of benchmarks/gpu_pcg_benchmark_3d.py);
  ext3d_sphere.npz gamma (from this package's sphere assembly) and the
                   reference E built from it;
  stress2d.npz     reduced SPD systems of the 2D sliver stress harness
                   (code/fast_solver_workbench.py:138-198, called piecewise)
                   with the reference solve_cpu_cg iterations and solutions.
The fixtures are inputs/outputs only; no reference source is copied.
"""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import scipy.sparse as sp

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]


def main(ref_root: str) -> None:
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    sys.path.insert(0, str(Path(ref_root) / "code"))
    sys.path.insert(0, str(REPO / "gpu-cutcell-navier-stokes_b200"))
    import bell_3d_core as bell
    import cut_spline_sbp as c1
    import fast_solver_backends as fsb
    import oblique_cut_sbp as ob

    # ---- 1D cut forms ----------------------------------------------------
    out = {}
    k = 0
    for n, p, frac in [(6, 3, 0.0), (6, 3, 0.35), (5, 2, 0.9), (4, 4, 0.5)]:
        b = c1.make_open_uniform_basis(n_elements=n, degree=p)
        m = c1.assemble_cut_matrices(b, left=b.h * frac)
        for name in ("H", "Q", "K", "H_background", "boundary_form", "left_trace", "right_trace"):
            out[f"c{k}_{name}"] = getattr(m, name)
        out[f"c{k}_meta"] = np.array([n, p, frac])
        out[f"c{k}_greville"] = b.greville
        k += 1
    out["count"] = np.array(k)
    np.savez_compressed(HERE / "cut1d.npz", **out)

    # ---- 3D extension on the reference bell ------------------------------
    geom = bell.Bell3DGeometry.from_grid(20, 1.0e-3)
    asm = bell.assemble_bell_3d(geom, n_elements=20, degree=2, with_flux=False)
    agg = bell.polynomial_preserving_extension_3d(asm)
    E = agg.E.tocsr()
    E.sort_indices()
    np.savez_compressed(
        HERE / "ext3d_bell.npz",
        n=20, p=2, gamma=asm.gamma, indptr=E.indptr, indices=E.indices, data=E.data,
        shape=np.array(E.shape), interior=agg.interior, small=agg.small_support,
        residual=agg.polynomial_residual,
    )

    # ---- 3D extension on a sphere gamma ---------------------------------
    from types import SimpleNamespace

    from cutcell_b200.cutgeom import SphereExteriorLevelSet
    from cutcell_b200.problem import build_problem

    n, p = 8, 3
    prob = build_problem(SphereExteriorLevelSet((0.5, 0.5, 0.5), 0.31), n, p)
    bases = tuple(c1.make_open_uniform_basis(n_elements=n, degree=p) for _ in range(3))
    gamma = prob.gamma
    fake = SimpleNamespace(
        bases=bases, degree=p, gamma=gamma, active=np.where(gamma > 0)[0], H=sp.diags(prob.h_cut_diag),
        n_full=gamma.size,
    )
    agg = bell.polynomial_preserving_extension_3d(fake)
    E = agg.E.tocsr()
    E.sort_indices()
    np.savez_compressed(
        HERE / "ext3d_sphere.npz",
        n=n, p=p, gamma=gamma, indptr=E.indptr, indices=E.indices, data=E.data, shape=np.array(E.shape),
        interior=agg.interior, small=agg.small_support, residual=agg.polynomial_residual,
    )

    # ---- 2D stress systems + reference CPU CG ----------------------------
    out = {}
    cases = [(4, 8, e) for e in (1e-5, 1e-4, 1e-3, 1e-2, 1e-1)] + [(4, 16, 1e-5), (3, 12, 1e-3)]
    for k, (p, n, eps) in enumerate(cases):
        bx = c1.make_open_uniform_basis(n_elements=n, degree=p)
        by = c1.make_open_uniform_basis(n_elements=n, degree=p)
        cut = ob.HalfPlaneCut.from_angle(0.0, bx.h * (1.0 - eps))
        mats = ob.assemble_oblique_cut_matrices(bx, by, cut, quadrature_order=max(24, 2 * p + 14))
        agg = ob.polynomial_preserving_oblique_extension(
            bx, by, mats, support_threshold=0.05, preserve_degree=p, active_tol=1.0e-100
        )
        phys = ob.pullback_oblique_2d(mats, agg.E)
        A = sp.csr_matrix(0.5 * ((phys.K + phys.H) + (phys.K + phys.H).T))
        rng = np.random.default_rng(12345 + 17 * n + p)
        b = rng.standard_normal(A.shape[0])
        x, rep = fsb.solve_cpu_cg(A, b, tol=1e-8, maxiter=5000, preconditioner="jacobi")
        out[f"s{k}_indptr"] = A.indptr
        out[f"s{k}_indices"] = A.indices
        out[f"s{k}_data"] = A.data
        out[f"s{k}_b"] = b
        out[f"s{k}_x"] = x
        out[f"s{k}_meta"] = np.array([p, n, eps, rep.iterations, rep.relative_residual, A.shape[0], A.nnz])
    out["count"] = np.array(len(cases))
    np.savez_compressed(HERE / "stress2d.npz", **out)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
    from oracle.build_ref import reference_root

    main(str(reference_root(sys.argv[1] if len(sys.argv) > 1 else None)))
