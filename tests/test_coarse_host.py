"""Host tables of the two-level preconditioner (no GPU): the 1D B-spline
refinement is exact, its bands reproduce it, the coarsening rule, and the
prolongation P selects the kept DOFs' rows of R1 (x) R1 (x) R1."""

from __future__ import annotations

import numpy as np
import pytest

from cutcell_b200.bspline import global_values, make_basis
from cutcell_b200.coarse import _bands, coarse_factor, prolongation, refinement_1d


@pytest.mark.parametrize("n,p,c", [(8, 3, 2), (32, 3, 4), (12, 2, 2), (16, 4, 4), (24, 3, 4)])
def test_refinement_is_exact(n, p, c):
    R = refinement_1d(n, p, c)
    fb, cb = make_basis(n, p), make_basis(n // c, p)
    x = np.random.default_rng(1).uniform(0.0, 1.0, 400)
    np.testing.assert_allclose(global_values(fb, x) @ R, global_values(cb, x), atol=1e-13)
    # partition of unity is kept and every coarse function refines into p + 1 .. (p + 1) c + 1 - p fine ones
    np.testing.assert_allclose(R.sum(axis=1), 1.0, atol=1e-13)
    assert R.shape == (n + p, n // c + p)


def test_bands_reproduce_refinement():
    R = refinement_1d(32, 3, 4)
    plo, pw, pval, rlo, rw, rval = _bands(R)
    nb, nbc = R.shape
    Rp = np.zeros_like(R)
    Rr = np.zeros_like(R)
    for x in range(nb):
        assert 0 <= plo[x] and plo[x] + pw <= nbc
        Rp[x, plo[x]:plo[x] + pw] = pval[x]
    for a in range(nbc):
        assert 0 <= rlo[a] and rlo[a] + rw <= nb
        Rr[rlo[a]:rlo[a] + rw, a] = rval[a]
    np.testing.assert_array_equal(Rp, R)
    np.testing.assert_array_equal(Rr, R)
    assert pw <= 4 and rw <= 13
    # padded to p + 1 for the device's unrolled prolongation
    plo4, pw4, pval4, *_ = _bands(R, 4)
    assert pw4 == 4 and np.all(plo4 + 4 <= nbc)
    for x in range(nb):
        np.testing.assert_array_equal(R[x, plo4[x]:plo4[x] + 4], pval4[x])
        assert np.count_nonzero(R[x]) == np.count_nonzero(pval4[x])


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("n,c", [(8, 2), (16, 2), (32, 4), (64, 8)])
def test_prolongation_rows_fit_degree_plus_one(n, c, p):
    R = refinement_1d(n, p, c)
    _bands(R, p + 1)  # raises if a fine row needs a wider band


def test_coarse_factor_rule():
    assert coarse_factor(8, 3) == 2
    assert coarse_factor(16, 3) == 2
    assert coarse_factor(24, 3) == 4
    assert coarse_factor(32, 3) == 4
    assert coarse_factor(64, 3) == 8
    with pytest.raises(ValueError):
        coarse_factor(7, 3)
    with pytest.raises(ValueError):
        refinement_1d(10, 3, 4)


def test_prolongation_rows_are_kept_dofs():
    from cutcell_b200.workloads import sphere_poisson

    prob, ext = sphere_poisson(8, 3, 0.31)
    P, R = prolongation(prob, ext, 2)
    nb = prob.n_basis
    full_of_red = np.asarray(ext.device_layout()["full_of_red"])
    assert P.shape == (ext.n_red, R.shape[1] ** 3)
    rng = np.random.default_rng(4)
    for j in rng.choice(ext.n_red, 20, replace=False):
        f = full_of_red[j]
        x, y, z = f % nb, (f // nb) % nb, f // (nb * nb)
        dense = np.einsum("c,b,a->cba", R[z], R[y], R[x]).ravel()
        np.testing.assert_allclose(P[j].toarray().ravel(), dense, atol=1e-15)


class _HostOp:
    """The two attributes patch_layout reads from an operator (no device)."""

    def __init__(self, prob, ext):
        self.problem, self.extension = prob, ext


@pytest.mark.parametrize("n,p", [(8, 3), (10, 2)])
def test_patch_tilings_cover_reduced_dofs_once(n, p):
    from cutcell_b200.learned import patch_layout
    from cutcell_b200.workloads import sphere_poisson

    prob, ext = sphere_poisson(n, p, 0.31)
    op = _HostOp(prob, ext)
    nb = prob.n_basis
    full_of_red = np.asarray(ext.device_layout()["full_of_red"])
    for shift in (0, 1, 2, 3):
        lay = patch_layout(op, shift)
        red = lay.red[lay.red >= 0]
        np.testing.assert_array_equal(np.sort(red), np.arange(ext.n_red))
        # lane l of patch k holds the DOF at origin + (l % 4, l // 4 % 4, l // 16)
        k, lane = np.nonzero(lay.red >= 0)
        f = full_of_red[lay.red[k, lane]]
        x, y, z = f % nb, (f // nb) % nb, f // (nb * nb)
        o = lay.origin[k]
        np.testing.assert_array_equal(x - o[:, 0], lane % 4)
        np.testing.assert_array_equal(y - o[:, 1], (lane // 4) % 4)
        np.testing.assert_array_equal(z - o[:, 2], lane // 16)


@pytest.mark.parametrize("p,device_its", [(3, 18), (2, 12), (4, 26)])
def test_twolevel_iteration_on_the_host(p, device_its):
    """The two-level step z = zc + 0.3 (B_0 + B_1 + B_2 + B_3) (r - A zc)
    restated with the oracle's assembled E^T A E (sphere, n = 8): flexible PCG
    reaches 1e-9 in the iterations the device takes at each degree (measured on
    a B200: 18 at p = 3, 12 at p = 2, 26 at p = 4), and its solution matches a
    direct solve to the accuracy a 1e-9 residual allows."""
    import scipy.linalg as sla
    import scipy.sparse.linalg as spla

    from cutcell_b200.learned import patch_layout
    from cutcell_b200.workloads import sphere_poisson
    from oracle.aggregation import restrict_spd
    from oracle.assembly import assemble_full

    prob, ext = sphere_poisson(8, p, 0.31)
    A = restrict_spd(assemble_full(prob), ext.E).tocsr()
    A = (0.5 * (A + A.T)).tocsr()
    b = np.asarray(ext.E.T @ prob.load)
    op = _HostOp(prob, ext)
    tilings = []
    for shift in (0, 1, 2, 3):
        groups = [row[row >= 0] for row in patch_layout(op, shift).red]
        tilings.append([(g, np.linalg.inv(A[g][:, g].toarray())) for g in groups])
    P, _ = prolongation(prob, ext, coarse_factor(8, p))
    keep = np.nonzero(np.diff(P.indptr))[0]
    Pk = P[:, keep]
    cf = sla.cho_factor((Pk.T @ A @ Pk).toarray())

    def M(r):
        zc = Pk @ sla.cho_solve(cf, Pk.T @ r)
        q = r - A @ zc
        w = np.zeros_like(r)
        for T in tilings:
            for g, inv in T:
                w[g] += inv @ q[g]
        return zc + 0.3 * w

    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    pv = z.copy()
    rz = r @ z
    bn = np.linalg.norm(b)
    its = 0
    for its in range(1, 200):
        Ap = A @ pv
        al = rz / (pv @ Ap)
        x += al * pv
        rold = r.copy()
        r -= al * Ap
        if np.linalg.norm(r) <= 1e-9 * bn:
            break
        z = M(r)
        beta = (r @ z - rold @ z) / rz
        rz = r @ z
        pv = z + beta * pv
    assert its == device_its, its
    x_ref = spla.spsolve(A.tocsc(), b)
    # a relative residual of 1e-9 bounds the relative error by cond(A) * 1e-9:
    # cond(A) is 1.2e3, 4.0e4 and 1.1e6 at p = 2, 3, 4 (errors 2e-7 at p = 3,
    # 1.6e-6 at p = 4)
    kappa = np.linalg.cond(A.toarray())
    assert np.linalg.norm(x - x_ref) <= 1e-9 * kappa * np.linalg.norm(x_ref)


class _AssembledOp(_HostOp):
    """An operator on the CPU whose apply is the oracle's assembled E^T A E."""

    def __init__(self, prob, ext, A):
        import torch

        super().__init__(prob, ext)
        self.A, self.device, self.n = A, torch.device("cpu"), ext.n_red

    def apply(self, v):
        import torch

        return torch.as_tensor(self.A @ v.numpy())


def test_twolevel_setup_data_on_the_host():
    """The arrays the device receives, built on the CPU by the product's own
    setup against the oracle's assembled E^T A E (sphere, n = 8, p = 3):
    CoarseLevel's P and explicit FP64 Ac^-1, the first tiling's probed
    inverses (symmetrised, BF16 as stored) and the extra tilings'
    (OverlapTiling, BF16).  Flexible PCG with z = zc + 0.3 sum_i B_i (r - A zc)
    from exactly those arrays takes the device's 18 iterations."""
    import torch

    from cutcell_b200.coarse import CoarseLevel, OverlapTiling
    from cutcell_b200.learned import DevicePatches, patch_blocks, patch_inverses, patch_layout
    from cutcell_b200.workloads import sphere_poisson
    from oracle.aggregation import restrict_spd
    from oracle.assembly import assemble_full

    prob, ext = sphere_poisson(8, 3, 0.31)
    A = restrict_spd(assemble_full(prob), ext.E).tocsr()
    A = (0.5 * (A + A.T)).tocsr()
    b = np.asarray(ext.E.T @ prob.load)
    op = _AssembledOp(prob, ext, A)
    cl = CoarseLevel(op)
    lay0 = patch_layout(op, 0)
    inv0 = patch_inverses(patch_blocks(op, DevicePatches(op, lay0)), lay0.red)
    inv0 = 0.5 * (inv0 + np.transpose(inv0, (0, 2, 1)))
    tilings = [(lay0.red, torch.as_tensor(inv0).to(torch.bfloat16).double().numpy())]
    for shift in (1, 2, 3):
        t = OverlapTiling(op, shift)
        tilings.append((t.dp.layout.red, t.inv.double().numpy()))
    minv = cl._t["minv"].numpy()
    P = cl.P.tocsr()

    def M(r):
        zc = P @ (minv @ (P.T @ r))
        q = r - A @ zc
        w = np.zeros_like(r)
        for red, inv in tilings:
            for k in range(red.shape[0]):
                m = red[k] >= 0
                g = red[k][m]
                w[g] += inv[k][np.ix_(m, m)] @ q[g]
        return zc + 0.3 * w

    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    pv = z.copy()
    rz = r @ z
    bn = np.linalg.norm(b)
    its = 0
    for its in range(1, 200):
        Ap = A @ pv
        al = rz / (pv @ Ap)
        x += al * pv
        rold = r.copy()
        r -= al * Ap
        if np.linalg.norm(r) <= 1e-9 * bn:
            break
        z = M(r)
        beta = (r @ z - rold @ z) / rz
        rz = r @ z
        pv = z + beta * pv
    assert its == 18, its
