"""Two-level patch preconditioner (preconditioner="twolevel") on the
sphere-cut p = 3 systems (needs a B200).

* The device-probed Galerkin operator Ac = P^T (E^T A E) P equals the one
  formed from the oracle's assembled E^T A E to 1e-10 (relative, max entry).
* The device flexible PCG needs the same iterations as a NumPy restatement of
  the same iteration (exact patch inverses and Ac from the assembled matrix)
  within max(2, 3 %).
* Its tol-1e-13 solution is within 1e-9 (relative L2) of the oracle CG's.
* It needs at most 0.3 of the iterations of the exact patch solves alone
  ("block"); measured with the default three extra tilings (offsets 1, 2, 3,
  omega 0.3) 18 / 128 at n = 8, 19 / 150 at n = 16 and 29 / 208 at n = 24.
* Every reduced DOF lies in exactly one patch of each tiling.
"""

from __future__ import annotations

import numpy as np
import pytest
import scipy.linalg as sla

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _twolevel_fcg_cpu(A, b, groups, P, tol, maxiter=5000, extra=(), omega=1.0):
    """Flexible PCG (Polak-Ribiere beta) with z = zc + B (r - A zc),
    zc = P Ac^-1 P^T r, B the exact inverses of A on the patch index groups
    (with extra tilings' groups: z = zc + omega (B_0 + B_1 + ...) (r - A zc)):
    the device iteration restated with the assembled matrix."""
    invs = [np.linalg.inv(A[idx][:, idx].toarray()) for idx in groups]
    invs_x = [[np.linalg.inv(A[idx][:, idx].toarray()) for idx in g] for g in extra]
    keep = np.nonzero(np.diff(P.tocsc().indptr))[0]
    Pk = P.tocsc()[:, keep]
    Ac = (Pk.T @ A @ Pk).toarray()
    cf = sla.cho_factor(0.5 * (Ac + Ac.T))

    def M(r):
        zc = Pk @ sla.cho_solve(cf, Pk.T @ r)
        q = r - A @ zc
        w = np.zeros_like(r)
        for idx, inv in zip(groups, invs):
            w[idx] = inv @ q[idx]
        if not invs_x:
            return zc + w
        for g, iv in zip(extra, invs_x):
            for idx, inv in zip(g, iv):
                w[idx] += inv @ q[idx]
        return zc + omega * w

    bn = np.linalg.norm(b)
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = z.copy()
    rz = r @ z
    for k in range(1, maxiter + 1):
        Ap = A @ p
        al = rz / (p @ Ap)
        x += al * p
        rold = r.copy()
        r -= al * Ap
        if np.linalg.norm(r) / bn <= tol:
            return x, k
        z = M(r)
        beta = (r @ z - rold @ z) / rz
        rz = r @ z
        p = z + beta * p
    return x, maxiter


def _system(n):
    from cutcell_b200.workloads import sphere_poisson
    from oracle.aggregation import restrict_spd
    from oracle.assembly import assemble_full

    prob, ext = sphere_poisson(n, 3, 0.31)
    A = restrict_spd(assemble_full(prob), ext.E).tocsr()
    A = (0.5 * (A + A.T)).tocsr()
    b = np.asarray(ext.E.T @ prob.load)
    return prob, ext, A, b


@pytest.mark.parametrize("n", [8, 16, 24])
def test_twolevel_matches_cpu_and_beats_block(torch_cuda, n):
    from cutcell_b200 import solve_spd
    from cutcell_b200.coarse import attach_coarse
    from cutcell_b200.learned import patch_layout
    from cutcell_b200.operator import CutCellOperator
    from oracle.pcg import cg_loop

    prob, ext, A, b = _system(n)
    op = CutCellOperator(prob, ext)
    try:
        cl = attach_coarse(op)
        keep = cl.keep
        Pk = cl.P.tocsc()[:, keep]
        Ac_ref = (Pk.T @ A @ Pk).toarray()
        assert np.abs(cl.Ac - Ac_ref).max() <= 1e-10 * np.abs(Ac_ref).max()
        x9, r9 = solve_spd(op, b, tol=1e-9, maxiter=5000, preconditioner="twolevel")
        assert r9.success, r9
        groups = [row[row >= 0] for row in patch_layout(op).red]
        extra = [[row[row >= 0] for row in patch_layout(op, t).red] for t in cl.shifts]
        # every reduced DOF in exactly one patch of each tiling
        for g in [groups] + extra:
            assert np.array_equal(np.sort(np.concatenate(g)), np.arange(ext.n_red))
        _, it_cpu = _twolevel_fcg_cpu(A, b, groups, cl.P, 1e-9, extra=extra, omega=cl.omega)
        assert abs(r9.iterations - it_cpu) <= max(2, 0.03 * it_cpu), (r9.iterations, it_cpu)
        x13, r13 = solve_spd(op, b, tol=1e-13, maxiter=5000, preconditioner="twolevel")
        assert r13.success, r13
        x_ref, _ = cg_loop(A, b, tol=1e-13, maxiter=50000)
        err = np.linalg.norm(x13 - x_ref) / np.linalg.norm(x_ref)
        assert err <= 1e-9, err
        _, rb = solve_spd(op, b, tol=1e-9, maxiter=5000, preconditioner="block")
        assert rb.success, rb
        print(f"n={n} factor={cl.factor} coarse={keep.size} twolevel {r9.iterations} (cpu {it_cpu}) "
              f"block {rb.iterations} err {err:.2e} {r9.device_ms:.2f} ms vs {rb.device_ms:.2f} ms")
        assert r9.iterations <= 0.3 * rb.iterations
    finally:
        op.close()


@pytest.mark.parametrize("p", [2, 4])
def test_twolevel_other_degrees(torch_cuda, p):
    """Degrees 2 and 4 (the prolongation unrolls p + 1 terms per axis): the
    two-level solve converges, matches the oracle's solution and needs fewer
    iterations than the exact patch solves alone."""
    from cutcell_b200 import solve_spd
    from cutcell_b200.operator import CutCellOperator
    from cutcell_b200.workloads import sphere_poisson
    from oracle.aggregation import restrict_spd
    from oracle.assembly import assemble_full
    from oracle.pcg import cg_loop

    prob, ext = sphere_poisson(8, p, 0.31)
    A = restrict_spd(assemble_full(prob), ext.E).tocsr()
    b = np.asarray(ext.E.T @ prob.load)
    op = CutCellOperator(prob, ext)
    try:
        x, r = solve_spd(op, b, tol=1e-12, maxiter=5000, preconditioner="twolevel")
        assert r.success, r
        x_ref, _ = cg_loop(A, b, tol=1e-13, maxiter=50000)
        assert np.linalg.norm(x - x_ref) <= 1e-8 * np.linalg.norm(x_ref)
        _, r9 = solve_spd(op, b, tol=1e-9, maxiter=5000, preconditioner="twolevel")
        _, rb = solve_spd(op, b, tol=1e-9, maxiter=5000, preconditioner="block")
        assert r9.success and rb.success
        print(f"p={p} n=8 twolevel {r9.iterations} block {rb.iterations}")
        assert r9.iterations < rb.iterations
    finally:
        op.close()
