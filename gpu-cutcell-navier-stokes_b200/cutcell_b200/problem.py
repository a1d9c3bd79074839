"""Host-side setup of aggregated cut-cell Poisson / screened-Poisson systems.

This mirrors the reference's assembly layer (``assemble_bell_3d``,
code/bell_3d_core.py:275-430, and ``solve_poisson_3d``,
code/cut_3d_sbp.py:387-503) for implicitly defined 3D domains, but produces
the element-structured description the matrix-free device operator consumes
instead of a global sparse matrix:

* uncut (full) elements keep only per-axis 1D blocks -- the element block is
  ``Mz (x) My (x) (a_m Mx + K~x) + Mz (x) K~y (x) Mx + K~z (x) My (x) Mx`` with
  ``K~ = a_k K + F``, where ``F`` carries the symmetric weak-penalty (Nitsche)
  box-face terms ``beta t t^T - s (t dt^T + dt t^T)`` of code/cut_3d_sbp.py:426-460
  (they share the Kronecker structure of the stiffness factor);
* cut elements carry one dense ``(p+1)^3 x (p+1)^3`` block, integrated on the
  clipped cell (volume + cut surface + box faces inside the cell).

DOFs are flattened x-fastest, ``(iz*ny + iy)*nx + ix``
(code/cut_3d_sbp.py:20-22, code/bell_3d_core.py:313-317); the local element
ordering is the same with ``p+1`` in place of ``n``.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from .bspline import OpenUniformBasis, element_matrices_1d, gauss_legendre01, local_values, make_basis
from .cutgeom import cut_cell_quadrature

SOLID, FULL, CUT = 0, 1, 2


@dataclass
class CutCellProblem:
    n_elements: int
    degree: int
    basis: OpenUniformBasis
    a_mass: float
    a_stiff: float
    nitsche: bool
    beta: float
    elem_type: np.ndarray  # (nz, ny, nx) int8
    M1: np.ndarray  # (n, p+1, p+1) 1D element mass (same on all axes)
    Kt1: np.ndarray  # (3, n, p+1, p+1) per-axis a_k K + F
    cut_ids: np.ndarray  # (ncut,) linear element index ((ez*n)+ey)*n+ex
    cut_mats: np.ndarray  # (ncut, P, P) dense element blocks
    h_cut_diag: np.ndarray  # (N_full,) diagonal of the fluid mass
    h_bg_diag: np.ndarray  # (N_full,) diagonal of the background mass
    load: np.ndarray  # (N_full,) right-hand side in the full space
    cut_fractions: np.ndarray  # (nz, ny, nx)
    extras: dict = field(default_factory=dict)

    @property
    def n_basis(self) -> int:
        return self.basis.n_basis

    @property
    def n_full(self) -> int:
        return self.n_basis**3

    @property
    def P(self) -> int:
        return (self.degree + 1) ** 3

    @property
    def gamma(self) -> np.ndarray:
        g = np.zeros(self.n_full)
        pos = self.h_bg_diag > 0
        g[pos] = self.h_cut_diag[pos] / self.h_bg_diag[pos]
        return g

    @property
    def min_cut_fraction(self) -> float:
        f = self.cut_fractions[self.elem_type == CUT]
        f = f[f > 0]
        return float(f.min()) if f.size else 1.0

    def element_rows(self, ex, ey, ez) -> np.ndarray:
        """Global DOF rows of elements (vectorised); shape (m, P)."""
        p1 = self.degree + 1
        nb = self.n_basis
        ex = np.atleast_1d(ex)[:, None, None, None]
        ey = np.atleast_1d(ey)[:, None, None, None]
        ez = np.atleast_1d(ez)[:, None, None, None]
        l = np.arange(p1)
        rows = ((ez + l[None, :, None, None]) * nb + (ey + l[None, None, :, None])) * nb + (
            ex + l[None, None, None, :]
        )
        return rows.reshape(rows.shape[0], -1)

    def full_element_blocks(self, ex, ey, ez) -> np.ndarray:
        """Dense blocks of full elements (for assembly and tests); (m, P, P)."""
        M = self.M1
        Kt = self.Kt1
        k3 = lambda a, b, c: np.einsum("mij,mkl,mab->mikajlb", a, b, c).reshape(a.shape[0], self.P, self.P)
        Mz, My, Mx = M[ez], M[ey], M[ex]
        return (
            k3(Mz, My, self.a_mass * Mx + Kt[0][ex])
            + k3(Mz, Kt[1][ey], Mx)
            + k3(Kt[2][ez], My, Mx)
        )

    def assemble_full_csr(self) -> sp.csr_matrix:
        """Global operator in the full space (COO -> CSR), symmetrised as in
        code/bell_3d_core.py:396-399."""
        ez, ey, ex = np.nonzero(self.elem_type == FULL)
        rows_l, cols_l, vals_l = [], [], []
        chunk = 4096
        for s in range(0, ex.size, chunk):
            sl = slice(s, s + chunk)
            B = self.full_element_blocks(ex[sl], ey[sl], ez[sl])
            R = self.element_rows(ex[sl], ey[sl], ez[sl])
            rows_l.append(np.repeat(R, self.P, axis=1).ravel())
            cols_l.append(np.tile(R, (1, self.P)).ravel())
            vals_l.append(B.ravel())
        n = self.n_elements
        cz, cy, cx = np.unravel_index(self.cut_ids, (n, n, n))
        if self.cut_ids.size:
            R = self.element_rows(cx, cy, cz)
            rows_l.append(np.repeat(R, self.P, axis=1).ravel())
            cols_l.append(np.tile(R, (1, self.P)).ravel())
            vals_l.append(self.cut_mats.ravel())
        N = self.n_full
        A = sp.coo_matrix(
            (np.concatenate(vals_l), (np.concatenate(rows_l), np.concatenate(cols_l))), shape=(N, N)
        ).tocsr()
        return ((A + A.T) * 0.5).tocsr()


def _face_matrix(basis: OpenUniformBasis, side: int, beta: float) -> np.ndarray:
    """1D weak-penalty face factor on the first (side=-1) or last (side=+1) element."""
    p = basis.degree
    e = 0 if side < 0 else basis.n_elements - 1
    x = 0.0 if side < 0 else 1.0
    N, D = local_values(basis, np.array([e]), np.array([x]))
    t, dt = N[0], D[0]
    return beta * np.outer(t, t) - side * (np.outer(t, dt) + np.outer(dt, t))


def manufactured_sine():
    """u = sin(pi x) sin(pi y) sin(pi z), f = -Lap u = 3 pi^2 u."""
    k = np.pi

    def u(x, y, z):
        return np.sin(k * x) * np.sin(k * y) * np.sin(k * z)

    def f(x, y, z):
        return 3.0 * k * k * np.sin(k * x) * np.sin(k * y) * np.sin(k * z)

    return u, f


def manufactured_sine_grad():
    """Gradient of u = sin(pi x) sin(pi y) sin(pi z)."""
    k = np.pi

    def g(x, y, z):
        sx, sy, sz = np.sin(k * x), np.sin(k * y), np.sin(k * z)
        cx, cy, cz = np.cos(k * x), np.cos(k * y), np.cos(k * z)
        return k * cx * sy * sz, k * sx * cy * sz, k * sx * sy * cz

    return g


def solution_errors(prob: "CutCellProblem", phi, alpha, u, grad_u, q: int | None = None) -> dict:
    """Relative L2, H1-seminorm and maximum errors of u_h = sum alpha_i B_i
    against (u, grad u) over the fluid domain, as solve_poisson_3d reports
    them (code/cut_3d_sbp.py:506-531): ||u_h - u|| / ||u||, ||grad(u_h - u)|| /
    ||grad u||, max|u_h - u| / max|u| over the quadrature nodes.  Uncut
    elements use a (p+3)^3 tensor Gauss rule, cut elements the cut-cell rule
    of the given order (default 2p+2)."""
    from .cutgeom import cut_cell_quadrature

    p, n, nb = prob.degree, prob.n_elements, prob.n_basis
    h = prob.basis.h
    q = q or 2 * p + 2
    A3 = np.asarray(alpha, dtype=float).reshape(nb, nb, nb)  # (z, y, x)
    acc = {"e2": 0.0, "u2": 0.0, "g2": 0.0, "gu2": 0.0, "emax": 0.0, "umax": 0.0}

    def add(pts, w, ex, ey, ez):
        Nx, Dx = local_values(prob.basis, np.full(len(w), ex), pts[:, 0])
        Ny, Dy = local_values(prob.basis, np.full(len(w), ey), pts[:, 1])
        Nz, Dz = local_values(prob.basis, np.full(len(w), ez), pts[:, 2])
        C = A3[ez : ez + p + 1, ey : ey + p + 1, ex : ex + p + 1]
        uh = np.einsum("cba,mc,mb,ma->m", C, Nz, Ny, Nx)
        gx = np.einsum("cba,mc,mb,ma->m", C, Nz, Ny, Dx)
        gy = np.einsum("cba,mc,mb,ma->m", C, Nz, Dy, Nx)
        gz = np.einsum("cba,mc,mb,ma->m", C, Dz, Ny, Nx)
        ue = u(pts[:, 0], pts[:, 1], pts[:, 2])
        ux, uy, uz = grad_u(pts[:, 0], pts[:, 1], pts[:, 2])
        acc["e2"] += float(np.sum(w * (uh - ue) ** 2))
        acc["u2"] += float(np.sum(w * ue**2))
        acc["g2"] += float(np.sum(w * ((gx - ux) ** 2 + (gy - uy) ** 2 + (gz - uz) ** 2)))
        acc["gu2"] += float(np.sum(w * (ux**2 + uy**2 + uz**2)))
        acc["emax"] = max(acc["emax"], float(np.max(np.abs(uh - ue))))
        acc["umax"] = max(acc["umax"], float(np.max(np.abs(ue))))

    xg, wg = gauss_legendre01(p + 3)
    Z, Y, X = np.meshgrid(xg, xg, xg, indexing="ij")
    W3 = (wg[:, None, None] * wg[None, :, None] * wg[None, None, :]).ravel() * h**3
    ref = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    for ez, ey, ex in zip(*np.nonzero(prob.elem_type == FULL)):
        add((np.array([ex, ey, ez]) + ref) * h, W3, ex, ey, ez)
    for lin in prob.cut_ids:
        ez, ey, ex = int(lin) // (n * n), (int(lin) // n) % n, int(lin) % n
        cq = cut_cell_quadrature(phi, np.array([ex, ey, ez]) * h, h, q, box_faces=False)
        if cq.wv.size:
            add(cq.xv, cq.wv, ex, ey, ez)
    return {
        "l2": np.sqrt(acc["e2"] / acc["u2"]),
        "h1": np.sqrt(acc["g2"] / acc["gu2"]),
        "linf": acc["emax"] / acc["umax"],
    }


def build_problem(
    phi,
    n_elements: int,
    degree: int,
    *,
    a_mass: float = 0.0,
    a_stiff: float = 1.0,
    nitsche: bool = True,
    beta_factor: float = 12.0,
    forcing=None,
    dirichlet=None,
    quad_order: int | None = None,
    subdiv: int = 1,
    keep_green: bool = False,
    load_order: int | None = None,
    native: bool | None = None,
) -> CutCellProblem:
    """Assemble the element-structured operator and load for ``{phi > 0}``.

    ``beta = beta_factor (p+1)^2 / h`` as in code/cut_3d_sbp.py:426.  Cut
    blocks use the order-``quad_order`` rules (default 3p+1: exact for the
    degree-6p mass integrand); loads use order ``load_order`` (default p+4).
    ``native`` selects libcutcell_setup.so (default: when it is built).  When
    ``nitsche`` is false only ``a_mass H + a_stiff K`` is assembled (the
    screened-Poisson proxy of benchmarks/gpu_pcg_benchmark_3d.py:49-57).
    """
    n = int(n_elements)
    p = int(degree)
    p1 = p + 1
    basis = make_basis(n, p)
    h = basis.h
    nb = basis.n_basis
    N = nb**3
    beta = beta_factor * p1 * p1 / h
    nu = 1.0 if nitsche else 0.0
    q = quad_order or (3 * p + 1)  # exact for the degree-6p mass integrand

    # --- element classification on the sub-cell corner grid -------------
    g = np.linspace(0.0, 1.0, n * subdiv + 1)
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    fc = phi(X, Y, Z)
    fmin = np.full((n, n, n), np.inf)
    fmax = np.full((n, n, n), -np.inf)
    for dz in range(subdiv + 1):
        for dy in range(subdiv + 1):
            for dx in range(subdiv + 1):
                blk = fc[dz :: subdiv, dy :: subdiv, dx :: subdiv][:n, :n, :n]
                fmin = np.minimum(fmin, blk)
                fmax = np.maximum(fmax, blk)
    etype = np.full((n, n, n), CUT, dtype=np.int8)
    etype[fmin >= 0.0] = FULL
    etype[fmax <= 0.0] = SOLID

    # --- 1D factors ------------------------------------------------------
    M1, K1 = element_matrices_1d(basis)
    Kt = np.stack([a_stiff * K1.copy() for _ in range(3)])
    if nitsche:
        for ax in range(3):
            Kt[ax, 0] += _face_matrix(basis, -1, beta)
            Kt[ax, n - 1] += _face_matrix(basis, +1, beta)

    # --- background and fluid mass diagonals ----------------------------
    dM = np.einsum("eii->ei", M1)  # (n, p1)
    cz, cy, cx = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    cz, cy, cx = cz.ravel(), cy.ravel(), cx.ravel()
    tmp = PseudoRows(n, p)
    rows_all = tmp.rows(cx, cy, cz)
    diag_all = (dM[cz][:, :, None, None] * dM[cy][:, None, :, None] * dM[cx][:, None, None, :]).reshape(-1, p1**3)
    h_bg = np.zeros(N)
    np.add.at(h_bg, rows_all.ravel(), diag_all.ravel())
    full_mask = etype.ravel() == FULL
    h_cut = np.zeros(N)
    np.add.at(h_cut, rows_all[full_mask].ravel(), diag_all[full_mask].ravel())

    # --- load on full elements (tensor Gauss) ---------------------------
    load = np.zeros(N)
    if forcing is not None:
        qg = p + 3
        xg, wg = gauss_legendre01(qg)
        e = np.repeat(np.arange(n), qg)
        xq = (e + np.tile(xg, n)) * h
        wq = np.tile(wg, n) * h
        Nq, _ = local_values(basis, e, xq)
        Nq = Nq.reshape(n, qg, p1)
        xq = xq.reshape(n, qg)
        wq = wq.reshape(n, qg)
        fe = np.nonzero(full_mask)[0]
        for s0 in range(0, fe.size, 2048):
            idx = fe[s0 : s0 + 2048]
            ex, ey, ez = cx[idx], cy[idx], cz[idx]
            F = forcing(
                xq[ex][:, None, None, :], xq[ey][:, None, :, None], xq[ez][:, :, None, None]
            )  # (m, qz, qy, qx)
            F = F * wq[ez][:, :, None, None] * wq[ey][:, None, :, None] * wq[ex][:, None, None, :]
            # one axis at a time (the four-operand einsum is a naive 7-deep loop)
            t = np.einsum("mcba,mai->mcbi", F, Nq[ex])
            t = np.einsum("mcbi,mbj->mcji", t, Nq[ey])
            vals = np.einsum("mcji,mck->mkji", t, Nq[ez])
            np.add.at(load, rows_all[idx].ravel(), vals.reshape(-1))
    # box-face Dirichlet data on full boundary elements
    if nitsche and dirichlet is not None:
        qg = p + 3
        xg, wg = gauss_legendre01(qg)
        for ax in range(3):
            for side in (-1, 1):
                eb = 0 if side < 0 else n - 1
                xb = 0.0 if side < 0 else 1.0
                Nb, Db = local_values(basis, np.array([eb]), np.array([xb]))
                avec = beta * Nb[0] - side * Db[0]  # (p1,)
                sel = full_mask & ((cx, cy, cz)[ax] == eb)
                idx = np.nonzero(sel)[0]
                if idx.size == 0:
                    continue
                others = [a for a in range(3) if a != ax]
                E = (cx, cy, cz)
                e0, e1 = E[others[0]][idx], E[others[1]][idx]
                x0 = (e0[:, None] + xg[None, :]) * h
                x1 = (e1[:, None] + xg[None, :]) * h
                N0, _ = local_values(basis, np.repeat(e0, qg), x0.ravel())
                N1, _ = local_values(basis, np.repeat(e1, qg), x1.ravel())
                N0 = N0.reshape(-1, qg, p1)
                N1 = N1.reshape(-1, qg, p1)
                coords = [None, None, None]
                coords[ax] = np.full((idx.size, 1, 1), xb)
                coords[others[0]] = x0[:, None, :]
                coords[others[1]] = x1[:, :, None]
                G = dirichlet(*coords) * (wg[None, :, None] * h) * (wg[None, None, :] * h)
                # G[m, q1, q0]; face coefficient fc[m, l1, l0]
                fcoef = np.einsum("mba,mbj,mai->mji", G, N1, N0)
                full3 = np.zeros((idx.size, p1, p1, p1))
                # local order (lz, ly, lx): place the axis vector on the face axis
                if ax == 0:
                    full3 = np.einsum("i,mkj->mkji", avec, fcoef)
                elif ax == 1:
                    full3 = np.einsum("j,mki->mkji", avec, fcoef)
                else:
                    full3 = np.einsum("k,mji->mkji", avec, fcoef)
                np.add.at(load, rows_all[idx].ravel(), full3.reshape(-1))

    # --- cut elements ----------------------------------------------------
    cut_lin = np.nonzero(etype.ravel() == CUT)[0]
    P = p1**3
    fracs = np.zeros(n * n * n)
    fracs[full_mask] = 1.0
    ql = load_order or (p + 4)
    use_native = (native is None and not keep_green and _setup_lib() is not None) or native is True
    green = None
    if use_native:
        cut_mats, mdiag, vols, cload, keep = _cut_blocks_native(
            fc, subdiv, n, p, q, ql, cut_lin, basis, a_mass, a_stiff, nitsche, beta, forcing, dirichlet
        )
        fracs[cut_lin] = vols / h**3
        rows = rows_all[cut_lin]
        np.add.at(h_cut, rows.ravel(), mdiag.ravel())
        np.add.at(load, rows.ravel(), cload.ravel())
    else:
        cut_mats = np.zeros((cut_lin.size, P, P))
        green = {"Q": [np.zeros((cut_lin.size, P, P)) for _ in range(3)], "S": [np.zeros((cut_lin.size, P, P)) for _ in range(3)]} if keep_green else None
        keep = np.ones(cut_lin.size, dtype=bool)
        for k, lin in enumerate(cut_lin):
            ez, ey, ex = np.unravel_index(lin, (n, n, n))
            lo = np.array([ex, ey, ez], dtype=float) * h
            cq = cut_cell_quadrature(phi, lo, h, q, subdiv=subdiv, box_faces=nitsche or keep_green)
            fracs[lin] = cq.volume / h**3
            if cq.wv.size == 0:
                keep[k] = False
                continue
            phi_v, grad_v = _tensor_local(basis, ex, ey, ez, cq.xv)
            Wv = cq.wv
            Mloc = (phi_v * Wv[:, None]).T @ phi_v
            Kloc = sum((grad_v[d] * Wv[:, None]).T @ grad_v[d] for d in range(3))
            A = a_mass * Mloc + a_stiff * Kloc
            if cq.ws.size and (nitsche or keep_green):
                phi_s, grad_s = _tensor_local(basis, ex, ey, ez, cq.xs)
                Ws = cq.ws
                if nitsche:
                    dn = sum(grad_s[d] * cq.ns[:, d : d + 1] for d in range(3))
                    Nloc = (phi_s * Ws[:, None]).T @ dn
                    Mb = (phi_s * Ws[:, None]).T @ phi_s
                    A = A - Nloc - Nloc.T + beta * Mb
                if keep_green:
                    for d in range(3):
                        green["S"][d][k] = (phi_s * (Ws * cq.ns[:, d])[:, None]).T @ phi_s
            if keep_green:
                for d in range(3):
                    green["Q"][d][k] = (phi_v * Wv[:, None]).T @ grad_v[d]
            cut_mats[k] = 0.5 * (A + A.T)
            rows = rows_all[lin]
            np.add.at(h_cut, rows, np.diag(Mloc))
            if forcing is not None or (nitsche and dirichlet is not None):
                cl = cut_cell_quadrature(phi, lo, h, ql, subdiv=subdiv, box_faces=nitsche)
                if forcing is not None and cl.wv.size:
                    pv, _ = _tensor_local(basis, ex, ey, ez, cl.xv)
                    fv = forcing(cl.xv[:, 0], cl.xv[:, 1], cl.xv[:, 2])
                    np.add.at(load, rows, pv.T @ (cl.wv * fv))
                if nitsche and dirichlet is not None and cl.ws.size:
                    ps, gs = _tensor_local(basis, ex, ey, ez, cl.xs)
                    dnl = sum(gs[d] * cl.ns[:, d : d + 1] for d in range(3))
                    gv = dirichlet(cl.xs[:, 0], cl.xs[:, 1], cl.xs[:, 2])
                    np.add.at(load, rows, (beta * ps - dnl).T @ (cl.ws * gv))
    if not keep.all():
        # zero-volume cells carry nothing; treat them as solid
        for lin in cut_lin[~keep]:
            etype.ravel()[lin] = SOLID
        cut_lin = cut_lin[keep]
        cut_mats = cut_mats[keep]
        if green is not None:
            for key in ("Q", "S"):
                green[key] = [a[keep] for a in green[key]]
    prob = CutCellProblem(
        n_elements=n,
        degree=p,
        basis=basis,
        a_mass=float(a_mass),
        a_stiff=float(a_stiff),
        nitsche=bool(nitsche),
        beta=float(beta),
        elem_type=etype,
        M1=M1,
        Kt1=Kt,
        cut_ids=cut_lin.astype(np.int64),
        cut_mats=cut_mats,
        h_cut_diag=h_cut,
        h_bg_diag=h_bg,
        load=load,
        cut_fractions=fracs.reshape(n, n, n),
    )
    if green is not None:
        prob.extras["green"] = green
    return prob


class PseudoRows:
    """Row helper usable before the problem object exists."""

    def __init__(self, n: int, p: int):
        self.n = n
        self.p = p

    def rows(self, ex, ey, ez):
        p1 = self.p + 1
        nb = self.n + self.p
        l = np.arange(p1)
        ex = np.asarray(ex)[:, None, None, None]
        ey = np.asarray(ey)[:, None, None, None]
        ez = np.asarray(ez)[:, None, None, None]
        r = ((ez + l[None, :, None, None]) * nb + (ey + l[None, None, :, None])) * nb + (ex + l[None, None, None, :])
        return r.reshape(r.shape[0], -1)


def _tensor_local(basis: OpenUniformBasis, ex: int, ey: int, ez: int, X: np.ndarray):
    """Local 3D basis values (m, P) and gradients [3 x (m, P)] on one element."""
    p1 = basis.degree + 1
    m = X.shape[0]
    Nx, Dx = local_values(basis, np.full(m, ex), X[:, 0])
    Ny, Dy = local_values(basis, np.full(m, ey), X[:, 1])
    Nz, Dz = local_values(basis, np.full(m, ez), X[:, 2])
    t = lambda a, b, c: (a[:, :, None, None] * b[:, None, :, None] * c[:, None, None, :]).reshape(m, p1**3)
    return t(Nz, Ny, Nx), [t(Nz, Ny, Dx), t(Nz, Dy, Nx), t(Dz, Ny, Nx)]


_SETUP = None


def _setup_lib():
    """libcutcell_setup.so (native host setup), or None when it is not built."""
    global _SETUP
    if _SETUP is None:
        import ctypes as C
        from pathlib import Path

        path = Path(__file__).resolve().parent / "libcutcell_setup.so"
        if not path.exists():
            _SETUP = False
            return None
        lib = C.CDLL(str(path))
        P = C.c_void_p
        lib.cutcell_setup_count.argtypes = [P, P, P]
        lib.cutcell_setup_load_points.argtypes = [P, P, P, P, P]
        lib.cutcell_setup_blocks.argtypes = [P, P, P, P, P, P, P, P, P]
        lib.cutcell_setup_threads.argtypes = [C.c_int]
        for f in (lib.cutcell_setup_count, lib.cutcell_setup_load_points, lib.cutcell_setup_blocks, lib.cutcell_setup_threads):
            f.restype = C.c_int
        _SETUP = lib
    return _SETUP or None


def _cut_blocks_native(fc, subdiv, n, p, q, ql, cut_lin, basis, a_mass, a_stiff, nitsche, beta, forcing, dirichlet):
    import ctypes as C

    from .cutgeom import tet_rule, tri_rule

    lib = _setup_lib()
    s1 = subdiv + 1
    ez, ey, ex = np.unravel_index(cut_lin, (n, n, n))
    cells = np.ascontiguousarray(np.stack([ex, ey, ez], axis=1).astype(np.int32))
    corner = np.empty((cut_lin.size, s1, s1, s1))
    for dz in range(s1):
        for dy in range(s1):
            for dx in range(s1):
                corner[:, dz, dy, dx] = fc[ez * subdiv + dz, ey * subdiv + dy, ex * subdiv + dx]
    corner = np.ascontiguousarray(corner.reshape(cut_lin.size, -1))
    knots = np.ascontiguousarray(basis.knots)

    def rule4(q_):
        x, w = tet_rule(q_)
        return np.ascontiguousarray(np.column_stack([x, w]))

    def rule3(q_):
        x, w = tri_rule(q_)
        return np.ascontiguousarray(np.column_stack([x, w]))

    tr, sr, trl, srl = rule4(q), rule3(q), rule4(ql), rule3(ql)

    class Desc(C.Structure):
        _fields_ = [(k, C.c_int32) for k in ("n_elements", "degree", "subdiv", "box_faces", "n_cells", "n_tet", "n_tri", "n_tet_load", "n_tri_load", "pad")] + [
            (k, C.c_void_p) for k in ("cells", "corner_phi", "knots", "tet_rule", "tri_rule", "tet_load", "tri_load")
        ] + [(k, C.c_double) for k in ("a_mass", "a_stiff", "nitsche", "beta")]

    d = Desc()
    d.n_elements, d.degree, d.subdiv, d.box_faces, d.n_cells = n, p, subdiv, int(bool(nitsche)), cut_lin.size
    d.n_tet, d.n_tri, d.n_tet_load, d.n_tri_load = tr.shape[0], sr.shape[0], trl.shape[0], srl.shape[0]
    d.cells, d.corner_phi, d.knots = cells.ctypes.data, corner.ctypes.data, knots.ctypes.data
    d.tet_rule, d.tri_rule, d.tet_load, d.tri_load = tr.ctypes.data, sr.ctypes.data, trl.ctypes.data, srl.ctypes.data
    d.a_mass, d.a_stiff, d.nitsche, d.beta = float(a_mass), float(a_stiff), 1.0 if nitsche else 0.0, float(beta)
    nc = cut_lin.size
    nv = np.zeros(nc, dtype=np.int64)
    ns = np.zeros(nc, dtype=np.int64)
    if lib.cutcell_setup_count(C.byref(d), nv.ctypes.data, ns.ctypes.data):
        raise RuntimeError("cutcell_setup_count failed")
    voff = np.concatenate([[0], np.cumsum(nv)]).astype(np.int64)
    soff = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    xv = np.zeros((max(int(voff[-1]), 1), 3))
    xs = np.zeros((max(int(soff[-1]), 1), 3))
    fvals = gvals = None
    if forcing is not None or (nitsche and dirichlet is not None):
        lib.cutcell_setup_load_points(C.byref(d), voff.ctypes.data, soff.ctypes.data, xv.ctypes.data, xs.ctypes.data)
        if forcing is not None:
            fvals = np.ascontiguousarray(forcing(xv[:, 0], xv[:, 1], xv[:, 2]), dtype=float)
        if nitsche and dirichlet is not None:
            gvals = np.ascontiguousarray(dirichlet(xs[:, 0], xs[:, 1], xs[:, 2]), dtype=float)
    P = (p + 1) ** 3
    blocks = np.zeros((nc, P, P))
    mdiag = np.zeros((nc, P))
    vols = np.zeros(nc)
    cload = np.zeros((nc, P))
    rc = lib.cutcell_setup_blocks(
        C.byref(d), voff.ctypes.data, soff.ctypes.data,
        None if fvals is None else fvals.ctypes.data, None if gvals is None else gvals.ctypes.data,
        blocks.ctypes.data, mdiag.ctypes.data, vols.ctypes.data, cload.ctypes.data,
    )
    if rc:
        raise RuntimeError("cutcell_setup_blocks failed")
    keep = vols > 0.0
    return blocks, mdiag, vols, cload, keep
