"""Mixed precision under sliver stress: 3D plane-cut boxes, p = 4, n = 16
(8,000 full DOFs), normals |g| / ||g|| with g ~ N(0, I) on the positive
octant, worst cut-cell fluid fraction 1e-5 .. 1e-1, N(0, 1) right-hand
sides (seed 12345).  FP64 matrix-free Jacobi-PCG against the oracle's CG on
the assembled E^T A E; FP32 / BF16 operator storage inside FP64 iterative
refinement against the FP64 solution.

Bars: at tol 1e-9 the FP64 iterations are within max(1, 2 %) of the
oracle's; solved to tol 1e-13, the FP64 solution is within 1e-9 (relative
L2) of the oracle's 1e-13 solution and the FP32 refinement within 1e-7;
BF16 refinement either meets the FP32 bar at tol 1e-9 or stops cleanly
(breakdown or stagnation, finite iterate)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS = [1e-5, 1e-3, 1e-1]


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _case(k, eps):
    from cutcell_b200.aggregation import build_extension
    from cutcell_b200.problem import build_problem
    from cutcell_b200.workloads import sliver_plane
    from oracle.aggregation import restrict_spd
    from oracle.assembly import assemble_full

    rng = np.random.default_rng(12345 + k)
    phi = sliver_plane(16, rng.standard_normal(3), eps)
    prob = build_problem(phi, 16, 4)
    ext = build_extension(prob.gamma, prob.basis, 4)
    A = restrict_spd(assemble_full(prob), ext.E).tocsr()
    b = np.random.default_rng(12345).standard_normal(ext.n_red)
    return prob, ext, A, b


@pytest.mark.parametrize("k,eps", list(enumerate(EPS)))
def test_sliver_stress_mixed_precision(torch_cuda, k, eps):
    from cutcell_b200 import solve_spd
    from cutcell_b200.operator import CutCellOperator
    from oracle.pcg import cg_loop

    prob, ext, A, b = _case(k, eps)
    assert abs(prob.min_cut_fraction / eps - 1.0) < 1e-6
    x_ref, rep_ref = cg_loop(A, b, tol=1e-13, maxiter=50000)
    _, rep_o = cg_loop(A, b, tol=1e-9, maxiter=50000)
    op = CutCellOperator(prob, ext)
    try:
        x, rep = solve_spd(op, b, tol=1e-9, maxiter=50000)
        assert rep.success, rep
        assert abs(rep.iterations - rep_o["iterations"]) <= max(1, 0.02 * rep_o["iterations"])
        x64, rep64 = solve_spd(op, b, tol=1e-13, maxiter=50000)
        assert rep64.success, rep64
        assert np.linalg.norm(x64 - x_ref) / np.linalg.norm(x_ref) < 1e-9
        x32, rep32 = solve_spd(op, b, tol=1e-13, maxiter=50000, precision="fp32-ir")
        assert rep32.success, rep32
        assert np.linalg.norm(x32 - x_ref) / np.linalg.norm(x_ref) < 1e-7
        x16, rep16 = solve_spd(op, b, tol=1e-9, maxiter=50000, precision="bf16-ir")
        if rep16.success:
            assert np.linalg.norm(x16 - x_ref) / np.linalg.norm(x_ref) < 1e-7
        else:
            assert rep16.message in ("CG breakdown: non-positive curvature", "maximum iterations reached")
            assert np.all(np.isfinite(x16))
    finally:
        op.close()
