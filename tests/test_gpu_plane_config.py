"""The plain CPU-runnable configuration on the device: 3D Poisson on [0,1]^3
cut by a plane whose normal is rotated 5 degrees from x, worst cut cell 0.15,
p = 3, n = 8 (about 1.3k unknowns), FP64 Jacobi-PCG to 1e-10.  Checked
against the oracle's CG (iterations within max(1, 2 %): the system needs
about 670 iterations, and round-off in the summation order shifts that by a
few) and by the L2 / H1 errors
against u = sin sin sin, which must equal the direct solve's to 1e-6
relative (the discretisation error is about 4e-5 in L2)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_plane_config_fp64(golden):
    import scipy.sparse.linalg as spla
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from cutcell_b200 import solve_spd
    from cutcell_b200.cutgeom import PlaneLevelSet
    from cutcell_b200.operator import CutCellOperator
    from cutcell_b200.problem import manufactured_sine, manufactured_sine_grad, solution_errors
    from cutcell_b200.workloads import plane_poisson
    from oracle.aggregation import restrict_spd
    from oracle.pcg import cg_loop

    prob, ext, c = plane_poisson(8)
    a = np.deg2rad(5.0)
    phi = PlaneLevelSet((np.cos(a), np.sin(a), 0.0), c)
    A = restrict_spd(prob.assemble_full_csr(), ext.E)
    b = np.asarray(ext.E.T @ prob.load)
    assert 1200 <= ext.n_red <= 1400
    _, rep_o = cg_loop(A, b, tol=1e-10, maxiter=20000)
    op = CutCellOperator(prob, ext)
    try:
        x, rep = solve_spd(op, b, tol=1e-10, maxiter=20000)
    finally:
        op.close()
    band = max(1, 0.02 * rep_o["iterations"])
    assert rep.success and abs(rep.iterations - rep_o["iterations"]) <= band
    xc, repc = solve_spd(A, b, tol=1e-10, maxiter=20000)  # CSR drop-in path
    assert repc.success and abs(repc.iterations - rep_o["iterations"]) <= band
    u, _ = manufactured_sine()
    g = manufactured_sine_grad()
    xd = spla.spsolve(A.tocsc(), b)
    ed = solution_errors(prob, phi, ext.E @ xd, u, g)
    for xs in (x, xc):
        e = solution_errors(prob, phi, ext.E @ xs, u, g)
        for k in ("l2", "h1"):
            assert abs(e[k] / ed[k] - 1.0) < 1e-6, (k, e[k], ed[k])
    assert ed["l2"] < 1e-4
