"""Periodic-hill setup (host): the x-y cut forms on the curved hill wall, their
aggregation and reduction, the periodic spanwise pieces and the sparse
Galerkin sample machinery -- ``Hill3D::build`` (cpp/include/cut/hill3d.h:95-171)
with ``assemble_hill_cut_2d`` / ``hill_fluid_quadrature`` /
``assemble_hill_wall_traces`` (cpp/include/cut/hill_cut2d.h:45-235) and
``cut2d_active_sets`` / ``cut2d_extension`` (cpp/include/cut/cut2d.h:208-392),
generalised to an ANISOTROPIC x-y grid of ``nex x ney`` elements (the
reference builds ``ne x ne`` only).  At ``nex == ney`` every form reproduces
the reference build (pinned against its own output in the tests).

Geometry: the fluid is ``{ y >= h(x) }`` of ``[0, Lx] x [0, Ly]``, mapped to the
unit square by ``x' = x / Lx, y' = y / Ly`` (wall ``hbar(x') = h(Lx x') / Ly``);
``physical=True`` carries the physical metric (gradients ``/Lx, /Ly``, volume
Jacobian ``Lx Ly``, physical wall arc length and normal), as the DNS does.
The unit square holds ``nex`` elements along x and ``ney`` along y.

Outputs (``HillSetup``): reduced 2D forms ``M2, Qx2, Qy2, K2, KN2`` (dense,
``nr x nr``), ``M2inv``; the periodic z forms ``Mz, Kz, Sz`` (circulant
``nz x nz``), ``Mzinv``; the sparse reduced sample rows ``phi, dpx, dpy``
(CSR ``n2q x nr``, sorted modes), 2D weights ``w2``; z tables ``Vz, dVz``
(``nzq x nz``), weights ``wz``.  Fields are ``FieldH`` arrays ``(nr, nz)``.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from .bspline import element_of, local_values, make_basis

# ---------------------------------------------------------------------------
# wall profile
# ---------------------------------------------------------------------------

# The benchmark hill as six cubic segments in xhat = 28 * (distance from the
# nearest crest), y/H = a + b u + c u^2 + d u^3 with u = xhat - BREAKS[s].  These
# are the reference's C2-repaired coefficients (cpp/include/cut/hill_geom.h:
# 30-37); the same numbers are needed to build the same wall.
BREAKS = (0.0, 9.0, 14.0, 20.0, 30.0, 40.0, 54.0)
CUBICS = (
    (1.0000000000000004, 1.5020812190951664e-15, 2.3904900851070415e-04, -7.557135858141106e-05),
    (0.9642714492836167, -1.4060957982077751e-02, -1.8013776731852192e-03, 6.642249618292267e-05),
    (0.8572350295664743, -2.7093047500234838e-02, -8.0504023044439350e-04, 5.910719772570910e-05),
    (0.6784624509778259, -3.0369952911172730e-02, 2.5888932860460340e-04, -7.663273788288154e-06),
    (0.3929885809383813, -2.7491148475546758e-02, 2.8991114957172600e-05, 2.2274667324788843e-05),
    (0.1432508750033985, -2.0228925978970975e-02, 6.9723113469980320e-04, 1.201452733618056e-06),
)


@dataclass(frozen=True)
class HillWall:
    """y = h(x) on the periodic cell [0, Lx] (lengths in hill heights)."""

    Lx: float = 9.0
    Ly: float = 3.036

    def _seg(self, xhat):
        s = np.searchsorted(np.asarray(BREAKS[1:]) + 1e-9, xhat, side="left")
        return np.minimum(s, 5)

    def h(self, x):
        x = np.asarray(x, dtype=float)
        xhat = 28.0 * np.minimum(x, self.Lx - x)
        s = self._seg(xhat)
        c = np.asarray(CUBICS)[s]
        u = xhat - np.asarray(BREAKS)[s]
        y = c[..., 0] + u * (c[..., 1] + u * (c[..., 2] + u * c[..., 3]))
        return np.where(xhat >= BREAKS[6] - 1e-12, 0.0, y)

    def hp(self, x):
        x = np.asarray(x, dtype=float)
        xhat = 28.0 * np.minimum(x, self.Lx - x)
        s = self._seg(xhat)
        c = np.asarray(CUBICS)[s]
        u = xhat - np.asarray(BREAKS)[s]
        dy = c[..., 1] + u * (2.0 * c[..., 2] + u * 3.0 * c[..., 3])
        sgn = np.where(x < 0.5 * self.Lx, 1.0, -1.0)
        return np.where(xhat >= BREAKS[6] - 1e-12, 0.0, 28.0 * dy * sgn)

    def kinks(self):
        ks = [0.5 * self.Lx]
        for b in BREAKS[1:]:
            xm = b / 28.0
            if xm < 0.5 * self.Lx:
                ks += [xm, self.Lx - xm]
        return sorted(ks)

    # unit-square wall
    def hbar(self, xp):
        return self.h(self.Lx * np.asarray(xp, dtype=float)) / self.Ly

    def hbarp(self, xp):
        return self.hp(self.Lx * np.asarray(xp, dtype=float)) * self.Lx / self.Ly

    def kinks_unit(self):
        return [k / self.Lx for k in self.kinks()]


def _gauss(q: int):
    """Gauss-Legendre nodes and weights on [-1, 1], nodes in DESCENDING order
    (the ordering of the reference's rule, so quadrature points, and with them
    the sample rows, come out in the same order)."""
    g, w = np.polynomial.legendre.leggauss(q)
    return g[::-1].copy(), w[::-1].copy()


def _crossings(wall: HillWall, xa: float, xb: float, yk: float, nscan: int = 24):
    """Roots of hbar(x) = yk in (xa, xb): sign-change scan, then 60 bisections
    (hill_cut2d.h:47-65)."""
    out = []
    xs = xa + (xb - xa) * np.arange(nscan + 1) / nscan
    g = wall.hbar(xs) - yk
    for i in range(1, nscan + 1):
        gp, gc = g[i - 1], g[i]
        if gp == 0.0 or gp * gc < 0.0:
            lo, hi, glo = xs[i - 1], xs[i], gp
            for _ in range(60):
                m = 0.5 * (lo + hi)
                gm = float(wall.hbar(m)) - yk
                if glo * gm <= 0.0:
                    hi = m
                else:
                    lo, glo = m, gm
            r = 0.5 * (lo + hi)
            if xa + 1e-12 < r < xb - 1e-12:
                out.append(r)
    return out


def _unique_sorted(v):
    v = sorted(v)
    out = [v[0]]
    for t in v[1:]:
        if abs(t - out[-1]) >= 1e-12:
            out.append(t)
    return out


def fluid_quadrature(wall: HillWall, nex: int, ney: int, p: int, q: int | None = None):
    """Height-function fluid rule on the unit square (hill_fluid_quadrature,
    hill_cut2d.h:68-101) on an nex x ney grid: per cell, x sub-panels split at
    wall kinks and at the wall's crossings of the cell's bottom and top, then
    per x node a y rule from max(y0, hbar(x)) to the cell top.  Returns x, y, w
    (unit-square coordinates), cell-major (iy outer, ix inner)."""
    q = q or max(12, 2 * p + 8)
    g, wg = _gauss(q)
    hx, hy = 1.0 / nex, 1.0 / ney
    ku = wall.kinks_unit()
    X, Y, W = [], [], []
    for iy in range(ney):
        y0, y1 = iy * hy, (iy + 1) * hy
        for ix in range(nex):
            x0, x1 = ix * hx, (ix + 1) * hx
            br = [x0, x1] + [k for k in ku if x0 + 1e-12 < k < x1 - 1e-12]
            br += _crossings(wall, x0, x1, y0) + _crossings(wall, x0, x1, y1)
            br = _unique_sorted(br)
            for xa, xb in zip(br[:-1], br[1:]):
                if xb <= xa:
                    continue
                hxs, mx = 0.5 * (xb - xa), 0.5 * (xb + xa)
                xp = mx + hxs * g
                wx = wg * hxs
                lower = np.maximum(y0, wall.hbar(xp))
                keep = lower < y1 - 1e-14
                for xv, wv, lo in zip(xp[keep], wx[keep], lower[keep]):
                    hys, my = 0.5 * (y1 - lo), 0.5 * (y1 + lo)
                    X.append(np.full(q, xv))
                    Y.append(my + hys * g)
                    W.append(wv * wg * hys)
    if not X:
        return np.zeros(0), np.zeros(0), np.zeros(0)
    return np.concatenate(X), np.concatenate(Y), np.concatenate(W)


# ---------------------------------------------------------------------------
# 2D tensor basis on the anisotropic unit square
# ---------------------------------------------------------------------------


@dataclass
class Basis2D:
    nex: int
    ney: int
    p: int

    def __post_init__(self):
        self.bx = make_basis(self.nex, self.p)
        self.by = make_basis(self.ney, self.p)
        self.nbx = self.nex + self.p
        self.nby = self.ney + self.p
        self.n = self.nbx * self.nby
        # tensor Greville points, row = iy * nbx + ix
        self.gx = np.tile(self.bx.greville, self.nby)
        self.gy = np.repeat(self.by.greville, self.nbx)

    def local(self, x, y):
        """Rows (m, (p+1)^2) and values / x-, y-derivatives of the local tensor
        functions at (x, y) (cut2d_point_basis / _grad, cut2d.h:431-458); x and
        y are clamped to [0, 1] as local_1d does."""
        x = np.clip(np.asarray(x, dtype=float), 0.0, 1.0)
        y = np.clip(np.asarray(y, dtype=float), 0.0, 1.0)
        ex, ey = element_of(self.bx, x), element_of(self.by, y)
        vx, dx = local_values(self.bx, ex, x)
        vy, dy = local_values(self.by, ey, y)
        p1 = self.p + 1
        ja, ia = np.meshgrid(np.arange(p1), np.arange(p1), indexing="ij")  # (ja, ia), ia fastest
        ja, ia = ja.ravel(), ia.ravel()
        rows = (ey[:, None] + ja[None, :]) * self.nbx + (ex[:, None] + ia[None, :])
        phi = vy[:, ja] * vx[:, ia]
        px = vy[:, ja] * dx[:, ia]
        py = dy[:, ja] * vx[:, ia]
        return rows, phi, px, py

    def poly(self, max_total: int) -> np.ndarray:
        """Tensor monomial coefficient rows x^sx y^sy, ordered by total degree
        then sx (cut2d_tensor_poly, cut2d.h:228-245)."""
        from .bspline import polynomial_coefficients

        cx = polynomial_coefficients(self.bx, max_total)
        cy = polynomial_coefficients(self.by, max_total)
        rows = []
        for tot in range(max_total + 1):
            for sx in range(tot + 1):
                rows.append(np.kron(cy[tot - sx], cx[sx]))
        return np.asarray(rows)


def _accumulate(n, rows, A, B, w):
    """Dense sum_q w_q A_q B_q^T over local rows (q, k): M[rows_a, rows_b].
    Points sharing a cell (same local rows) are summed by one matrix product
    per cell, then scattered."""
    M = np.zeros((n, n))
    key = rows[:, 0] * n + rows[:, -1]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    starts = np.concatenate(([0], np.where(np.diff(ks) != 0)[0] + 1))
    ends = np.concatenate((starts[1:], [ks.size]))
    for s0, s1 in zip(starts, ends):
        idx = order[s0:s1]
        r = rows[idx[0]]
        M[np.ix_(r, r)] += (A[idx] * w[idx, None]).T @ B[idx]
    return M


@dataclass
class HillForms2D:
    basis: Basis2D
    H: np.ndarray
    Qx: np.ndarray
    Qy: np.ndarray
    K: np.ndarray
    Hbg: np.ndarray
    Mw: np.ndarray
    Bn: np.ndarray
    quad: tuple  # unit-square fluid rule (x, y, w)


def hill_forms_2d(wall: HillWall, nex: int, ney: int, p: int, physical: bool, q: int | None = None) -> HillForms2D:
    """Volume forms H, Qx (phi_a dphi_b/dx), Qy, K, the background mass Hbg and
    the no-slip wall traces Mw, Bn (assemble_hill_cut_2d / assemble_hill_wall_
    traces, hill_cut2d.h:105-233)."""
    q = q or max(12, 2 * p + 8)
    B = Basis2D(nex, ney, p)
    Lx, Ly = (wall.Lx, wall.Ly) if physical else (1.0, 1.0)
    x, y, w = fluid_quadrature(wall, nex, ney, p, q)
    rows, phi, px, py = B.local(x, y)
    px, py = px / Lx, py / Ly
    wj = w * Lx * Ly
    n = B.n
    H = _accumulate(n, rows, phi, phi, wj)
    Qx = _accumulate(n, rows, phi, px, wj)
    Qy = _accumulate(n, rows, phi, py, wj)
    K = _accumulate(n, rows, px, px, wj) + _accumulate(n, rows, py, py, wj)
    # background tensor mass with the same Jacobian (gamma classifier)
    from .bspline import element_matrices_1d

    def full_mass(b):
        Me, _ = element_matrices_1d(b, max(8, p + 4))
        M = np.zeros((b.n_basis, b.n_basis))
        for e in range(b.n_elements):
            M[e : e + p + 1, e : e + p + 1] += Me[e]
        return M

    Hbg = Lx * Ly * np.kron(full_mass(B.by), full_mass(B.bx))
    # wall traces: curved bottom (split at kinks and x cell edges) and flat top
    g, wg = _gauss(q)
    br = _unique_sorted([0.0, 1.0] + [k for k in wall.kinks_unit() if 1e-12 < k < 1 - 1e-12]
                        + [e / nex for e in range(1, nex)])
    xs, ws = [], []
    for xa, xb in zip(br[:-1], br[1:]):
        if xb <= xa:
            continue
        hh, mm = 0.5 * (xb - xa), 0.5 * (xb + xa)
        xs.append(mm + hh * g)
        ws.append(wg * hh)
    xw, ww = np.concatenate(xs), np.concatenate(ws)
    yw, hpw = wall.hbar(xw), wall.hbarp(xw)
    Lp = np.sqrt(Lx * Lx + (Ly * hpw) ** 2)
    r1, ph1, dx1, dy1 = B.local(xw, yw)
    Mw = _accumulate(n, r1, ph1, ph1, Lp * ww)
    dn = (Ly / Lx) * hpw[:, None] * dx1 - (Lx / Ly) * dy1
    Bn = _accumulate(n, r1, dn, ph1, ww)
    bt = [e / nex for e in range(nex + 1)]
    xt = np.concatenate([0.5 * (b - a) * g + 0.5 * (b + a) for a, b in zip(bt[:-1], bt[1:])])
    wt = np.concatenate([0.5 * (b - a) * wg for a, b in zip(bt[:-1], bt[1:])])
    r2, ph2, dx2, dy2 = B.local(xt, np.ones_like(xt))
    Mw += _accumulate(n, r2, ph2, ph2, Lx * wt)
    Bn += _accumulate(n, r2, (Lx / Ly) * dy2, ph2, wt)
    return HillForms2D(B, H, Qx, Qy, K, Hbg, Mw, Bn, (x, y, w))


def active_sets(f: HillForms2D, support_threshold: float = 0.05, active_tol: float = 1e-22):
    """gamma = diag(H) / diag(Hbg) and the active / interior / small sets
    (cut2d_active_sets, cut2d.h:210-220)."""
    bg = np.diag(f.Hbg)
    gamma = np.where(bg > 0.0, np.diag(f.H) / np.where(bg > 0.0, bg, 1.0), 0.0)
    active = np.where(gamma > active_tol)[0]
    interior = np.where(gamma >= support_threshold)[0]
    small = active[gamma[active] < support_threshold]
    return gamma, active, interior, small


def _max_total_degree(n_interior: int) -> int:
    m = 0
    while (m + 1) * (m + 2) // 2 <= n_interior:
        m += 1
    return m - 1


def extension_2d(f: HillForms2D, gamma, interior, small, preserve_degree: int | None = None) -> np.ndarray:
    """The polynomial-preserving 2D extension (cut2d_extension, cut2d.h:305-392):
    identity columns for the interior modes; each small mode is reproduced from
    the interior modes of the smallest Chebyshev index neighbourhood whose
    locally scaled monomial block has full row rank (all |R_dd| > 1e-9 of its
    QR), by the minimum-norm solution.  Local scaling: monomials of
    ((x - x_b) / hx, (y - y_b) / hy)."""
    from math import comb

    B = f.basis
    n, nbx = B.n, B.nbx
    n_int = interior.size
    deg = min(B.p if preserve_degree is None else preserve_degree, _max_total_degree(n_int))
    poly = B.poly(deg)
    powers = [(sx, tot - sx) for tot in range(deg + 1) for sx in range(tot + 1)]
    nt = len(powers)
    col = np.full(n, -1)
    col[interior] = np.arange(n_int)
    E = np.zeros((n, n_int))
    E[interior, np.arange(n_int)] = 1.0
    hx, hy = 1.0 / B.nex, 1.0 / B.ney
    ix_int, iy_int = interior % nbx, interior // nbx
    for b in small:
        ibx, iby = b % nbx, b // nbx
        xb, yb = B.gx[b], B.gy[b]
        T = np.zeros((nt, nt))
        for kr, (P, Q) in enumerate(powers):
            scale = 1.0 / (hx**P * hy**Q)
            for kc, (I, J) in enumerate(powers):
                if I <= P and J <= Q:
                    T[kr, kc] = scale * comb(P, I) * comb(Q, J) * (-xb) ** (P - I) * (-yb) ** (Q - J)
        pl = T @ poly
        target = pl[:, b]
        cheb = np.maximum(np.abs(ix_int - ibx), np.abs(iy_int - iby))
        cand = None
        for radius in range(0, max(B.nbx, B.nby) + 1):
            c = interior[cheb <= radius]
            if c.size < nt:
                continue
            R = np.linalg.qr(pl[:, c].T, mode="r")
            cand = c
            if np.min(np.abs(np.diag(R))) > 1e-9:
                break
        if cand is None or cand.size < nt:
            continue
        C = pl[:, cand]
        Qm, Rm = np.linalg.qr(C.T)
        z = np.linalg.solve(Rm.T, target) if np.all(np.abs(np.diag(Rm)) > 1e-300) else np.linalg.lstsq(Rm.T, target, rcond=None)[0]
        E[b, col[cand]] = Qm @ z
    return E


def periodic_forms(nz: int, p: int, Lz: float):
    """Circulant mass M_ij = int N_i N_j, derivative K_ij = int N_i N_j' and
    stiffness S_ij = int N_i' N_j' of the periodic cardinal B-splines
    N_i(z) = beta_p((z - i hz) / hz) on [0, Lz] (assemble_forms_periodic,
    cpp/include/core/bspline.h:401-416), by Gauss rules exact on every knot
    panel."""
    hz = Lz / nz
    zq, wq = periodic_quadrature(nz, p, Lz, q=p + 4)
    V, dV = periodic_basis(nz, p, Lz, zq)
    M = (V.T * wq) @ V
    K = (V.T * wq) @ dV
    S = (dV.T * wq) @ dV
    return M, K, S


def _cardinal(p: int, t):
    """Centered cardinal B-spline of degree p and its derivative at t (support
    [-(p+1)/2, (p+1)/2]), from the uniform Cox-de Boor recursion."""
    t = np.asarray(t, dtype=float)
    u = t + 0.5 * (p + 1)

    def N(k, u):
        # N_{0,k}(u) on integer knots 0..k+1
        vals = [((u >= j) & (u < j + 1)).astype(float) for j in range(k + 1)]
        for d in range(1, k + 1):
            vals = [((u - j) / d) * vals[j] + ((j + d + 1 - u) / d) * vals[j + 1] for j in range(k + 1 - d)]
        return vals[0]

    val = N(p, u)
    der = N(p - 1, u) - N(p - 1, u - 1.0)
    return val, der


def periodic_basis(nz: int, p: int, Lz: float, z):
    """V[q, i] = N_i(z_q), dV[q, i] = N_i'(z_q), wrapped to the nearest image
    (PeriodicZ::basis / dbasis, hill3d.h:37-47)."""
    hz = Lz / nz
    z = np.asarray(z, dtype=float)
    d = z[:, None] - np.arange(nz)[None, :] * hz
    d = d - Lz * np.floor(d / Lz + 0.5)
    v, dv = _cardinal(p, d / hz)
    return v, dv / hz


def periodic_quadrature(nz: int, p: int, Lz: float, q: int | None = None):
    """Per-element Gauss rule of order p + 6 on [0, Lz] (Hill3D::build, :158-163)."""
    q = q or p + 6
    g, wg = _gauss(q)
    hz = Lz / nz
    e = np.repeat(np.arange(nz), q)
    z = (e + 0.5) * hz + 0.5 * hz * np.tile(g, nz)
    w = 0.5 * hz * np.tile(wg, nz)
    return z, w


@dataclass
class HillSetup:
    nex: int
    ney: int
    p: int
    nz: int
    Lz: float
    physical: bool
    wall: HillWall
    forms: HillForms2D
    E: np.ndarray
    interior: np.ndarray
    gamma: np.ndarray
    M2: np.ndarray
    Qx2: np.ndarray
    Qy2: np.ndarray
    K2: np.ndarray
    KN2: np.ndarray
    M2inv: np.ndarray
    Mz: np.ndarray
    Kz: np.ndarray
    Sz: np.ndarray
    Mzinv: np.ndarray
    phi: sp.csr_matrix
    dpx: sp.csr_matrix
    dpy: sp.csr_matrix
    w2: np.ndarray
    xq: np.ndarray  # unit-square quadrature coordinates of the 2D points
    yq: np.ndarray
    Vz: np.ndarray
    dVz: np.ndarray
    wz: np.ndarray
    zq: np.ndarray
    extra: dict = field(default_factory=dict)

    @property
    def nr(self) -> int:
        return self.M2.shape[0]

    @property
    def n2q(self) -> int:
        return self.w2.size

    @property
    def nzq(self) -> int:
        return self.wz.size

    def machinery(self) -> dict:
        """The inputs of HillAdvection / the oracle's skew_conv."""
        return {"phi": self.phi, "dpx": self.dpx, "dpy": self.dpy, "w2": self.w2, "Vz": self.Vz, "dVz": self.dVz,
                "wz": self.wz, "M2inv": self.M2inv, "Mzinv": self.Mzinv}


def sample_rows(B: Basis2D, E: np.ndarray, x, y, Lx: float = 1.0, Ly: float = 1.0):
    """Reduced sample / gradient rows (CSR, n_points x n_red) at unit-square
    points; gradients in the physical metric (1/Lx, 1/Ly)."""
    rows, ph, px, py = B.local(x, y)
    npt, k = rows.shape
    Ec = sp.csr_matrix(E)
    ip, ic, iv = Ec.indptr, Ec.indices, Ec.data
    b = rows.reshape(-1)
    cnt = ip[b + 1] - ip[b]
    tot = int(cnt.sum())
    off = np.arange(tot) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    src = np.repeat(ip[b], cnt) + off
    m = ic[src]
    e = iv[src]
    q = np.repeat(np.repeat(np.arange(npt), k), cnt)
    nr = E.shape[1]
    key = q.astype(np.int64) * nr + m
    order = np.argsort(key, kind="stable")
    ks = key[order]
    starts = np.concatenate(([0], np.where(np.diff(ks) != 0)[0] + 1)) if ks.size else np.zeros(0, int)
    vals = []
    for v in (ph, px / Lx, py / Ly):
        c = np.repeat(v.reshape(-1), cnt) * e
        vals.append(np.add.reduceat(c[order], starts) if ks.size else np.zeros(0))
    uk = ks[starts]
    keep = (vals[0] != 0.0) | (vals[1] != 0.0) | (vals[2] != 0.0)
    uk = uk[keep]
    qi, mi = uk // nr, uk % nr
    ptr = np.concatenate(([0], np.cumsum(np.bincount(qi, minlength=npt))))
    mk = lambda v: sp.csr_matrix((v[keep], mi, ptr), shape=(npt, nr))
    return mk(vals[0]), mk(vals[1]), mk(vals[2])


def build_hill(nex: int, ney: int, p: int = 3, nz: int = 32, Lz: float = 4.5, *, physical: bool = False,
               wall: HillWall | None = None, penalty_beta: float = 10.0) -> HillSetup:
    """Hill3D::build (hill3d.h:95-171) on an nex x ney x-y grid.  The no-slip
    penalty uses beta = penalty_beta p^2 over the wall-normal cell size
    (Ly / ney physical, 1 / ney on the unit square; the reference's ne)."""
    wall = wall or HillWall()
    f = hill_forms_2d(wall, nex, ney, p, physical)
    gamma, active, interior, small = active_sets(f)
    E = extension_2d(f, gamma, interior, small)
    pb = lambda A: E.T @ A @ E
    M2, Qx2, Qy2, K2 = pb(f.H), pb(f.Qx), pb(f.Qy), pb(f.K)
    Mw2, Bn2 = pb(f.Mw), pb(f.Bn)
    hcell = (wall.Ly / ney) if physical else (1.0 / ney)
    beta = penalty_beta * p * p
    KN2 = K2 - Bn2 - Bn2.T + (beta / hcell) * Mw2
    M2inv = np.linalg.inv(M2)
    Mz, Kz, Sz = periodic_forms(nz, p, Lz)
    Mzinv = np.linalg.inv(Mz)
    # sparse reduced sample rows: for each 2D point, every local function's
    # E row, accumulated per reduced mode in local-function order and kept
    # where any of the three values is nonzero, modes ascending (Hill3D::build,
    # hill3d.h:130-154)
    x, y, w = f.quad
    Lx, Ly = (wall.Lx, wall.Ly) if physical else (1.0, 1.0)
    phi, dpx, dpy = sample_rows(f.basis, E, x, y, Lx, Ly)
    w2 = w * (Lx * Ly)
    zq, wz = periodic_quadrature(nz, p, Lz)
    Vz, dVz = periodic_basis(nz, p, Lz, zq)
    return HillSetup(nex, ney, p, nz, Lz, physical, wall, f, E, interior, gamma, M2, Qx2, Qy2, K2, KN2, M2inv,
                     Mz, Kz, Sz, Mzinv, phi, dpx, dpy, w2, x, y, Vz, dVz, wz, zq)


# ---------------------------------------------------------------------------
# fields on the hill: L2 projection, weak divergence, initial condition
# ---------------------------------------------------------------------------


def sample_2d(hs: HillSetup, c):
    """(n2q, nz) values of a FieldH at the 2D points."""
    return hs.phi @ c


def l2_project(hs: HillSetup, fq):
    """hill_l2_project (hill3d.h:276-287): the Galerkin load of a quadrature
    field fq (n2q, nzq) followed by the separable mass solve."""
    t = (fq * hs.wz[None, :]) @ hs.Vz  # (n2q, nz)
    red = hs.phi.T @ (hs.w2[:, None] * t)
    return hs.M2inv @ red @ hs.Mzinv.T


def weak_div(hs: HillSetup, ux, uy, uz):
    """hill_weak_div (hill3d.h:330-334): Qx2 ux Mz^T + Qy2 uy Mz^T + M2 uz Kz^T
    (FieldH arrays, z applies along the second axis)."""
    return hs.Qx2 @ ux @ hs.Mz.T + hs.Qy2 @ uy @ hs.Mz.T + hs.M2 @ uz @ hs.Kz.T


def parabolic_ic(hs: HillSetup, *, ub: float = 1.0, amp: float = 0.01, seed: int = 20260629):
    """Initial velocity of the channel step: u_x = 6 U_b eta (1 - eta) with
    eta = (y - h(x)) / (Ly - h(x)) the local wall-normal coordinate (bulk
    U_b in every column), L2-projected onto the reduced space (hill_l2_project),
    plus a uniform random perturbation amp U_b U(-0.5, 0.5) on every
    coefficient of all three components (numpy default_rng(seed)); u_y = u_z
    start from the perturbation alone."""
    hb = hs.wall.hbar(hs.xq)
    eta = np.clip((hs.yq - hb) / np.maximum(1.0 - hb, 1e-300), 0.0, 1.0)
    prof = 6.0 * ub * eta * (1.0 - eta)
    # the profile is constant in z, so its z load is one row (wz^T Vz) and
    # the projection is separable: no (n2q, nzq) field is formed
    red = hs.phi.T @ (hs.w2 * prof)
    ux = np.outer(hs.M2inv @ red, hs.Mzinv @ (hs.wz @ hs.Vz))
    rng = np.random.default_rng(seed)
    shape = (hs.nr, hs.nz)
    ux = ux + amp * ub * rng.uniform(-0.5, 0.5, shape)
    uy = amp * ub * rng.uniform(-0.5, 0.5, shape)
    uz = amp * ub * rng.uniform(-0.5, 0.5, shape)
    return ux, uy, uz
