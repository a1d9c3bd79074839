"""Batched persistent Jacobi-PCG on the device (cutcell_batch_* through the C ABI).

Parity: every system of a batch against the oracle's Jacobi-PCG (same
algorithm, FP64) and, for the oblique golden systems, against the
reference's own solve_cpu_cg solutions (tests/golden/oblique2d.npz).
Bar: iterations within max(2, 5 %) of the oracle, true relative residual
<= 10 tol, solution within 1e-6 (relative L2) of the oracle's at tol 1e-9.
The iteration band is wider than for the single-system tests because the
dot products of a team of C CTAs are summed in a C-dependent order, and CG
on the p = 3..5 B-spline mass matrices (clustered spectra) shifts by a few
iterations under such round-off changes (seen: 101 vs 104 at C = 4).
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu

TOL = 1e-9


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="module")
def golden_systems(golden):
    z = np.load(golden / "oblique2d.npz")
    out = []
    for k in range(int(z["count"])):
        for form in ("mass", "stiffness"):
            pre = f"c{k}_{form}"
            A = sp.csr_matrix((z[f"{pre}_data"], z[f"{pre}_indices"], z[f"{pre}_indptr"]))
            out.append((A, z[f"{pre}_b"], z[f"{pre}_x"], int(z[f"{pre}_rep"][0])))
    return out


@pytest.fixture(scope="module")
def sample_systems():
    from cutcell_b200 import oblique2d as ob

    cases = [c for c in ob.sample_cases(72) if c[0] <= 12][:14]
    systems = [ob.build_oblique(*c).A for c in cases]
    rng = np.random.default_rng(5)
    rhs = [rng.standard_normal(A.shape[0]) for A in systems]
    return systems, rhs


def _band(it):
    return max(2, 0.05 * it)


def _oracle(A, b):
    from oracle.pcg import cg_loop

    return cg_loop(A, b, tol=TOL, maxiter=20000)


def _check(results, systems, rhs, oracle=None):
    for i, ((x, rep), A, b) in enumerate(zip(results, systems, rhs)):
        xo, ro = oracle[i] if oracle else _oracle(A, b)
        assert rep.success, (i, rep)
        assert rep.relative_residual <= 10 * TOL
        assert abs(rep.iterations - ro["iterations"]) <= _band(ro["iterations"]), (i, rep.iterations, ro)
        assert np.linalg.norm(x - xo) / np.linalg.norm(xo) < 1e-6, i


@pytest.mark.parametrize("cluster", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("staging", ["none", "full"])
def test_golden_systems_all_shapes(torch_cuda, golden_systems, cluster, staging):
    from cutcell_b200.batch import BatchConfig, solve_batch

    systems = [g[0] for g in golden_systems]
    rhs = [g[1] for g in golden_systems]
    res = solve_batch(systems, rhs, tol=TOL, maxiter=20000, config=BatchConfig(cluster=cluster, staging=staging))
    _check(res, systems, rhs)
    for (x, rep), (_, _, xr, it_ref) in zip(res, golden_systems):
        # the reference's own SciPy CG at the same tolerance
        assert abs(rep.iterations - it_ref) <= _band(it_ref)
        assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-6


def test_uneven_sample_with_autotune(torch_cuda, sample_systems):
    from cutcell_b200.batch import BatchSolver

    systems, rhs = sample_systems
    bs = BatchSolver(systems)
    try:
        bs.rhs.copy_(torch_cuda.from_numpy(bs.packed.pack(rhs)))
        best = bs.autotune(tol=TOL, maxiter=20000, reps=1, clusters=(1, 2, 4))
        assert bs.config == best and bs.tuning
        assert all(np.isfinite(t) for _, t in bs.tuning[:1])
        res = bs.solve(rhs, tol=TOL, maxiter=20000)
        _check(res, systems, rhs)
        # same configuration, same bits
        res2 = bs.solve(rhs, tol=TOL, maxiter=20000)
        for (x1, r1), (x2, r2) in zip(res, res2):
            np.testing.assert_array_equal(x1, x2)
            assert r1.iterations == r2.iterations
    finally:
        bs.close()


def test_matches_single_system_device_solver(torch_cuda, sample_systems):
    from cutcell_b200 import solve_spd
    from cutcell_b200.batch import BatchConfig, solve_batch

    systems, rhs = sample_systems
    res = solve_batch(systems[:6], rhs[:6], tol=TOL, maxiter=20000, config=BatchConfig(cluster=2, staging="half"))
    for (x, rep), A, b in zip(res, systems[:6], rhs[:6]):
        xs, rs = solve_spd(A, b, tol=TOL, maxiter=20000)
        assert rs.success and rep.success
        assert abs(rep.iterations - rs.iterations) <= _band(rs.iterations)
        assert np.linalg.norm(x - xs) / np.linalg.norm(xs) < 1e-6


def test_edge_cases(torch_cuda):
    """1x1 and 2x2 systems, a zero right-hand side, maxiter 0, no
    preconditioner, and a system with more CTAs than rows."""
    from cutcell_b200 import _lib
    from cutcell_b200.batch import BatchConfig, BatchSolver

    A1 = sp.csr_matrix(np.array([[4.0]]))
    A2 = sp.csr_matrix(np.array([[2.0, -1.0], [-1.0, 2.0]]))
    A3 = sp.csr_matrix(sp.diags([-1.0, 2.5, -1.0], [-1, 0, 1], shape=(50, 50)))
    systems = [A1, A2, A3, A3]
    rhs = [np.array([2.0]), np.array([1.0, 0.0]), np.zeros(50), np.ones(50)]
    bs = BatchSolver(systems, config=BatchConfig(cluster=8, staging="full"))
    try:
        res = bs.solve(rhs, tol=TOL, maxiter=1000)
        np.testing.assert_allclose(res[0][0], [0.5], rtol=1e-15)
        np.testing.assert_allclose(res[1][0], [2.0 / 3.0, 1.0 / 3.0], rtol=1e-12)
        # b = 0: p.Ap = 0 at the first step, reported as a breakdown with x = 0,
        # as solve_gpu_cg does (code/fast_solver_backends.py:251-256)
        assert not res[2][1].success and not res[2][0].any()
        assert res[2][1].message == "CG breakdown: non-positive curvature" and res[2][1].iterations == 1
        assert res[3][1].success
        res = bs.solve(rhs, tol=TOL, maxiter=0)
        assert res[3][1].message == "maximum iterations reached" and res[3][1].iterations == 0
        res = bs.solve(rhs, tol=TOL, maxiter=1000, preconditioner="none")
        assert [r.success for _, r in res] == [True, True, False, True]
        np.testing.assert_allclose(res[1][0], [2.0 / 3.0, 1.0 / 3.0], rtol=1e-12)
        with pytest.raises(ValueError):
            bs.solve(rhs, preconditioner="jacobi+learned")
    finally:
        bs.close()
    with pytest.raises(_lib.CutcellLibraryError):
        BatchSolver([A3], config=BatchConfig(cluster=3))


def test_malformed_system_reports_shape_error(torch_cuda):
    """A column index out of range marks only that system (status E_SHAPE);
    the others still solve."""
    from cutcell_b200.batch import BatchConfig, BatchSolver

    good = sp.csr_matrix(sp.diags([-1.0, 3.0, -1.0], [-1, 0, 1], shape=(20, 20)))
    bad = good.copy()
    bs = BatchSolver([good, bad, good], config=BatchConfig(cluster=2, staging="none"))
    try:
        # corrupt one column index of system 1 on the device
        start = good.nnz
        bs.indices[start + 5] = 999
        rhs = [np.ones(20)] * 3
        res = bs.solve(rhs, tol=TOL, maxiter=1000)
        assert res[0][1].success and res[2][1].success
        assert not res[1][1].success and res[1][1].message == "inconsistent sizes"
    finally:
        bs.close()
