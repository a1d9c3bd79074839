"""2D oblique half-plane cut systems (host setup for batched solves).

Restates the reference's 2D cut-cell pipeline for a unit square cut by the
half-plane ``normal . x >= offset``:

* cell clipping and Duffy/Gauss quadrature of the clipped polygon
  (code/oblique_cut_sbp.py:117-238);
* cut-domain forms H, K, Qx, Qy, Sx, Sy (code/oblique_cut_sbp.py:271-433;
  DOF index ``ix + (n+p) * iy``);
* active sets and the polynomial-preserving extension E
  (code/oblique_cut_sbp.py:574-672);
* the pullback ``E^T M E`` (code/oblique_cut_sbp.py:693-707) and the
  symmetrised reduced systems of the stress harness
  (code/fast_solver_workbench.py:138-198: ``0.5 (A + A^T)`` with
  ``A = K + H`` for the stiffness form, ``A = H`` for the mass form).

Every cell, cut or not, is integrated by the clipped-polygon rule of the
given order (the square itself is two Duffy triangles), as in the reference:
at the default order max(10, p + 5) that rule is not exact for p = 5
products, and the forms follow the rule, not the exact integrals.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from functools import lru_cache

import numpy as np
import scipy.sparse as sp

from .bspline import OpenUniformBasis, gauss_legendre01, local_values, make_basis, polynomial_coefficients

_INSIDE_TOL = 1.0e-14


@lru_cache(maxsize=None)
def _gl01(q: int):
    return gauss_legendre01(q)


def default_quadrature_order(p: int) -> int:
    """Default clipped-cell rule of assemble_oblique_cut_matrices (code/oblique_cut_sbp.py:286)."""
    return max(10, p + 5)


def clip_polygon(poly: np.ndarray, normal: np.ndarray, offset: float) -> np.ndarray:
    """Sutherland-Hodgman clip of a CCW polygon to ``normal . x >= offset``
    (code/oblique_cut_sbp.py:117-147): inside tolerance 1e-14, the crossing
    parameter clamped to [0, 1], coincident neighbours (within 1e-13) merged."""
    if len(poly) == 0:
        return np.empty((0, 2))
    dots = [float(np.dot(normal, v)) for v in poly]
    f = [d - offset for d in dots]
    ins = [d >= offset - _INSIDE_TOL for d in dots]
    pts = []
    m = len(poly)
    for k in range(m):
        j = k - 1  # previous vertex (wraps to the last one)
        if ins[k]:
            if not ins[j]:
                pts.append(_crossing(poly[j], poly[k], f[j], f[k]))
            pts.append(poly[k].copy())
        elif ins[j]:
            pts.append(_crossing(poly[j], poly[k], f[j], f[k]))
    out = []
    for q in pts:
        if not out or np.linalg.norm(q - out[-1]) > 1.0e-13:
            out.append(q)
    if len(out) > 1 and np.linalg.norm(out[0] - out[-1]) <= 1.0e-13:
        out.pop()
    return np.asarray(out, dtype=float).reshape(-1, 2)


def _crossing(a, b, fa, fb):
    den = fa - fb
    if abs(den) < 1.0e-30:
        return 0.5 * (a + b)
    t = min(1.0, max(0.0, fa / den))
    return a + t * (b - a)


def polygon_area(poly: np.ndarray) -> float:
    if len(poly) < 3:
        return 0.0
    x, y = poly[:, 0], poly[:, 1]
    return float(0.5 * np.sum(x * np.roll(y, -1) - y * np.roll(x, -1)))


def triangle_rule(v0, v1, v2, q: int):
    """Collapsed (Duffy) q x q Gauss rule on a triangle: point
    ``v0 + u e1 + (1-u) v e2``, weight ``|det| (1-u) w_u w_v``."""
    u, wu = _gl01(q)
    e1, e2 = v1 - v0, v2 - v0
    det = abs(float(e1[0] * e2[1] - e1[1] * e2[0]))
    U, V = np.meshgrid(u, u, indexing="ij")
    WU, WV = np.meshgrid(wu, wu, indexing="ij")
    om = 1.0 - U
    pts = v0[None, :] + U.reshape(-1, 1) * e1[None, :] + (om * V).reshape(-1, 1) * e2[None, :]
    return pts[:, 0], pts[:, 1], (det * om * WU * WV).ravel()


def polygon_rule(poly: np.ndarray, q: int):
    """Fan triangulation from the first vertex, each triangle by ``triangle_rule``."""
    if polygon_area(poly) < 0.0:
        poly = poly[::-1]
    parts = [triangle_rule(poly[0], poly[k], poly[k + 1], q) for k in range(1, len(poly) - 1)]
    return tuple(np.concatenate([p[i] for p in parts]) for i in range(3))


def edge_rule(a, b, q: int):
    """q-point Gauss rule on segment a->b with the right-hand normal (dy, -dx)."""
    g, w = _gl01(q)
    d = b - a
    length = float(np.linalg.norm(d))
    pts = a[None, :] + g[:, None] * d[None, :]
    normal = np.zeros(2) if length <= 1.0e-15 else np.array([d[1], -d[0]]) / length
    return pts[:, 0], pts[:, 1], length * w, normal


def _interval_forms(basis: OpenUniformBasis):
    """Exact 1D element mass, stiffness and advection ``C[i,j] = int N_i N_j'``,
    shape (n_elements, p+1, p+1)."""
    p, ne, h = basis.degree, basis.n_elements, basis.h
    xg, wg = gauss_legendre01(p + 2)
    e = np.repeat(np.arange(ne), xg.size)
    x = (e + np.tile(xg, ne)) * h
    w = (np.tile(wg, ne) * h).reshape(ne, -1)
    N, D = local_values(basis, e, x)
    N = N.reshape(ne, xg.size, p + 1)
    D = D.reshape(ne, xg.size, p + 1)
    M = np.einsum("eqi,eq,eqj->eij", N, w, N)
    K = np.einsum("eqi,eq,eqj->eij", D, w, D)
    Cm = np.einsum("eqi,eq,eqj->eij", N, w, D)
    return M, K, Cm


@dataclass
class ObliqueForms:
    """Cut-domain forms on the full (n+p)^2 tensor space (dense)."""

    basis: OpenUniformBasis
    normal: np.ndarray
    offset: float
    H: np.ndarray
    K: np.ndarray
    Qx: np.ndarray
    Qy: np.ndarray
    Sx: np.ndarray
    Sy: np.ndarray
    hbg_diag: np.ndarray

    @property
    def gamma(self) -> np.ndarray:
        g = np.zeros(self.H.shape[0])
        d = np.diag(self.H)
        pos = self.hbg_diag > 0.0
        g[pos] = d[pos] / self.hbg_diag[pos]
        return g


def assemble_forms(n: int, p: int, normal, offset: float, q: int | None = None) -> ObliqueForms:
    """H, K, Qx, Qy, Sx, Sy of the cut square (code/oblique_cut_sbp.py:271-379)."""
    basis = make_basis(n, p)
    q = q or default_quadrature_order(p)
    normal = np.asarray(normal, dtype=float)
    nb = basis.n_basis
    nf = nb * nb
    h = basis.h
    H = np.zeros((nf, nf))
    K = np.zeros((nf, nf))
    Qx = np.zeros((nf, nf))
    Qy = np.zeros((nf, nf))
    Sx = np.zeros((nf, nf))
    Sy = np.zeros((nf, nf))
    M1, K1, C1 = _interval_forms(basis)
    loc = np.arange(p + 1)

    def rows_of(ix, iy):
        return ((iy + loc)[:, None] * nb + (ix + loc)[None, :]).ravel()

    def tensor_at(ix, iy, x, y):
        Nx, Dx = local_values(basis, np.full(x.size, ix), x)
        Ny, Dy = local_values(basis, np.full(y.size, iy), y)
        phi = (Ny.T[:, None, :] * Nx.T[None, :, :]).reshape(-1, x.size)
        px = (Ny.T[:, None, :] * Dx.T[None, :, :]).reshape(-1, x.size)
        py = (Dy.T[:, None, :] * Nx.T[None, :, :]).reshape(-1, x.size)
        return phi, px, py

    def on_boundary(a, b):
        mid = 0.5 * (a + b)
        on_cut = abs(float(mid @ normal - offset)) <= 1.0e-10
        on_box = min(abs(mid[0]), abs(mid[0] - 1.0), abs(mid[1]), abs(mid[1] - 1.0)) <= 1.0e-12
        return on_cut or on_box

    for iy in range(n):
        for ix in range(n):
            cell = np.array([[ix * h, iy * h], [(ix + 1) * h, iy * h], [(ix + 1) * h, (iy + 1) * h], [ix * h, (iy + 1) * h]])
            poly = clip_polygon(cell, normal, offset)
            if len(poly) < 3 or abs(polygon_area(poly)) <= 1.0e-16:
                continue
            if polygon_area(poly) < 0.0:
                poly = poly[::-1]
            x, y, w = polygon_rule(poly, q)
            phi, px, py = tensor_at(ix, iy, x, y)
            r = rows_of(ix, iy)
            idx = np.ix_(r, r)
            pw = phi * w
            H[idx] += pw @ phi.T
            Qx[idx] += pw @ px.T
            Qy[idx] += pw @ py.T
            K[idx] += (px * w) @ px.T + (py * w) @ py.T
            for k in range(len(poly)):
                a, b = poly[k], poly[(k + 1) % len(poly)]
                if not on_boundary(a, b):
                    continue
                x, y, w, nrm = edge_rule(a, b, q)
                if not nrm.any():
                    continue
                phi, _, _ = tensor_at(ix, iy, x, y)
                r = rows_of(ix, iy)
                idx = np.ix_(r, r)
                bm = (phi * w) @ phi.T
                Sx[idx] += nrm[0] * bm
                Sy[idx] += nrm[1] * bm
    m1 = np.zeros(nb)
    for e in range(n):
        m1[e : e + p + 1] += np.diag(M1[e])
    hbg = np.kron(m1, m1)
    return ObliqueForms(basis, normal, float(offset), H, K, Qx, Qy, Sx, Sy, hbg)


@dataclass
class ObliqueExtension:
    E: np.ndarray  # dense (n_full, n_red)
    interior: np.ndarray
    small_support: np.ndarray
    active: np.ndarray
    gamma: np.ndarray
    degree: int
    polynomial_residual: float


def monomial_rows_2d(basis: OpenUniformBasis, degree: int) -> np.ndarray:
    """Coefficient rows of x^r y^s, r + s <= degree, ordered by total degree then
    r ascending (code/oblique_cut_sbp.py:596-611); entry ``iy*nb + ix``."""
    c = polynomial_coefficients(basis, degree)
    return np.asarray([np.kron(c[t - r], c[r]) for t in range(degree + 1) for r in range(t + 1)])


def build_extension_2d(
    forms: ObliqueForms, support_threshold: float = 0.05, degree: int | None = None, active_tol: float = 1.0e-22
) -> ObliqueExtension:
    """Polynomial-preserving extension (code/oblique_cut_sbp.py:574-672).

    Interior functions (gamma >= threshold) get identity columns.  Each small
    active function takes the least-squares (minimum-norm) weights that
    reproduce every total-degree monomial from its nearest interior
    neighbours by Greville distance (ties in interior order), the neighbour
    set grown one at a time from the monomial count until the coefficient
    block has full rank (singular values above 1e-12).
    """
    basis = forms.basis
    gamma = forms.gamma
    active = np.where(gamma > active_tol)[0]
    interior = np.where(gamma >= support_threshold)[0]
    small = active[gamma[active] < support_threshold]
    if interior.size == 0:
        raise ValueError("no interior basis functions")
    req = basis.degree if degree is None else degree
    cap = 0
    while (cap + 1) * (cap + 2) // 2 <= interior.size:
        cap += 1
    deg = min(req, cap - 1)
    poly = monomial_rows_2d(basis, deg)
    nt = poly.shape[0]
    nf = gamma.size
    E = np.zeros((nf, interior.size))
    E[interior, np.arange(interior.size)] = 1.0
    col = np.full(nf, -1, dtype=np.int64)
    col[interior] = np.arange(interior.size)
    g = basis.greville
    gx, gy = np.meshgrid(g, g, indexing="xy")
    grev = np.column_stack([gx.ravel(), gy.ravel()])
    for b in small:
        dist = np.linalg.norm(grev[interior] - grev[b], axis=1)
        order = interior[np.argsort(dist, kind="stable")]
        chosen = order[:nt]
        for k in range(nt, order.size + 1):
            if np.linalg.matrix_rank(poly[:, order[:k]], tol=1.0e-12) == nt:
                chosen = order[:k]
                break
        w = np.linalg.lstsq(poly[:, chosen], poly[:, b], rcond=None)[0]
        E[b, col[chosen]] = w
    mask = gamma > active_tol
    res = max(float(np.linalg.norm(E @ row[interior] - row * mask, ord=np.inf)) for row in poly)
    return ObliqueExtension(E, interior, small, active, gamma, deg, res)


@dataclass
class ObliqueSystem:
    """One oblique-cut SPD system ``0.5 (A + A^T)`` on the reduced space."""

    n: int
    p: int
    angle: float  # radians
    offset: float
    form: str  # "mass" | "stiffness"
    A: sp.csr_matrix
    n_full: int
    meta: dict = field(default_factory=dict)

    @property
    def n_red(self) -> int:
        return self.A.shape[0]


def reduced_matrix(forms: ObliqueForms, ext: ObliqueExtension, form: str) -> sp.csr_matrix:
    if form == "mass":
        M = forms.H
    elif form == "stiffness":
        M = forms.K + forms.H
    else:
        raise ValueError(f"unknown form {form!r}")
    E = ext.E
    A = E.T @ M @ E
    A = sp.csr_matrix(0.5 * (A + A.T))
    A.sort_indices()
    return A


def build_oblique(
    n: int,
    p: int,
    angle: float,
    offset: float,
    form: str = "stiffness",
    quadrature_order: int | None = None,
    support_threshold: float = 0.05,
    active_tol: float = 1.0e-22,
) -> ObliqueSystem:
    """Cut the unit square by ``(cos a, sin a) . x >= offset`` (angle in radians)."""
    nrm = np.array([np.cos(angle), np.sin(angle)])
    nrm = nrm / np.linalg.norm(nrm)
    forms = assemble_forms(n, p, nrm, offset, quadrature_order)
    ext = build_extension_2d(forms, support_threshold, p, active_tol)
    A = reduced_matrix(forms, ext, form)
    meta = {"n_small": int(ext.small_support.size), "min_gamma": float(ext.gamma[ext.active].min())}
    return ObliqueSystem(n, p, float(angle), float(offset), form, A, forms.H.shape[0], meta)


def sample_cases(count: int = 72, seed: int = 20260629):
    """The batched-solve draw: angle ~ U[0, 45] degrees, offset ~ U(0, h),
    p ~ {3, 4, 5}, n ~ {6, 8, 12, 16, 24}, mass or stiffness with equal odds.
    Returns a list of (n, p, angle_rad, offset, form)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice([6, 8, 12, 16, 24]))
        p = int(rng.choice([3, 4, 5]))
        ang = float(np.deg2rad(rng.uniform(0.0, 45.0)))
        off = float(rng.uniform(0.0, 1.0))
        while off <= 0.0:
            off = float(rng.uniform(0.0, 1.0))
        form = "mass" if rng.uniform() < 0.5 else "stiffness"
        out.append((n, p, ang, off / n, form))
    return out
