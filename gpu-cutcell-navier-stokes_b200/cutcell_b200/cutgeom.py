"""Cut-cell volume and surface quadrature for implicit 3D geometries (host setup).

The physical domain is ``{phi > 0}`` inside the unit box.  Each background cell
(optionally split into ``s^3`` sub-cells) is divided into the six Kuhn
tetrahedra (one per axis permutation; the split is conforming between
neighbouring cells), ``phi`` is interpolated linearly on every tetrahedron and
the tetrahedron is clipped by the half-space ``phi_lin >= 0``.  This is the 3D
lift of the reference's 2D half-plane pipeline -- Sutherland-Hodgman clip,
fan triangulation, collapsed-coordinate (Duffy) Gauss rules
(code/oblique_cut_sbp.py:121-248) -- with tetrahedra in place of triangles:

* a clipped tetrahedron is a tetrahedron or a prism, split into <= 3
  tetrahedra, each integrated by the conical product rule (Gauss-Jacobi in the
  two collapsed directions, Gauss-Legendre in the last; exact for total degree
  ``2q-1``);
* the zero set inside a tetrahedron is a triangle or a quad (two triangles),
  integrated by the collapsed triangle rule; its outward normal is
  ``-grad(phi_lin)/|grad(phi_lin)|``;
* tetrahedron faces on the box boundary are clipped the same way and carry the
  box face normal.

For a plane ``phi`` the linear interpolation is exact, so plane cuts are
integrated exactly (the 3D counterpart of ``assemble_oblique_cut_matrices``,
code/oblique_cut_sbp.py:271-433).  For a sphere the geometry is the piecewise
linear interpolant of the signed distance on the sub-cell grid; the Green
identity ``Q + Q^T = S`` then holds to round-off on that discrete geometry.
"""

from __future__ import annotations

from dataclasses import dataclass
from itertools import permutations

import numpy as np
from scipy.special import roots_jacobi


# ---------------------------------------------------------------------------
# Level sets: the fluid is {phi > 0}.
# ---------------------------------------------------------------------------


@dataclass(frozen=True)
class PlaneLevelSet:
    """Half-space ``normal . x >= offset`` (the 3D ``HalfPlaneCut``,
    code/oblique_cut_sbp.py:17-28)."""

    normal: tuple[float, float, float]
    offset: float

    def __call__(self, x, y, z):
        n = np.asarray(self.normal, dtype=float)
        n = n / np.linalg.norm(n)
        return n[0] * x + n[1] * y + n[2] * z - self.offset


@dataclass(frozen=True)
class SphereExteriorLevelSet:
    """The unit box minus a ball: ``phi = |x - c| - r`` (signed distance)."""

    center: tuple[float, float, float]
    radius: float

    def __call__(self, x, y, z):
        c = self.center
        return np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2) - self.radius


# ---------------------------------------------------------------------------
# Reference rules.
# ---------------------------------------------------------------------------


def _jacobi01(q: int, alpha: int) -> tuple[np.ndarray, np.ndarray]:
    """Gauss-Jacobi on [0,1] for the weight (1-s)^alpha."""
    x, w = roots_jacobi(q, alpha, 0)
    return 0.5 * (x + 1.0), w / 2.0 ** (alpha + 1)


def tet_rule(q: int) -> tuple[np.ndarray, np.ndarray]:
    """Conical product rule on the unit simplex; barycentric (a,b,c) and weights
    summing to 1/6.  Exact for total degree <= 2q-1."""
    s1, w1 = _jacobi01(q, 2)
    s2, w2 = _jacobi01(q, 1)
    s3, w3 = _jacobi01(q, 0)
    A, B, C = np.meshgrid(s1, s2, s3, indexing="ij")
    W = w1[:, None, None] * w2[None, :, None] * w3[None, None, :]
    a = A
    b = (1.0 - A) * B
    c = (1.0 - A) * (1.0 - B) * C
    return np.stack([a.ravel(), b.ravel(), c.ravel()], axis=1), W.ravel()


def tri_rule(q: int) -> tuple[np.ndarray, np.ndarray]:
    """Collapsed rule on the unit triangle; weights summing to 1/2."""
    s1, w1 = _jacobi01(q, 1)
    s2, w2 = _jacobi01(q, 0)
    A, B = np.meshgrid(s1, s2, indexing="ij")
    W = w1[:, None] * w2[None, :]
    return np.stack([A.ravel(), ((1.0 - A) * B).ravel()], axis=1), W.ravel()


# Kuhn split of the unit cube: vertex k of tet pi is sum of the first k unit
# vectors in the order pi.
_CUBE_CORNERS = np.array([[i & 1, (i >> 1) & 1, (i >> 2) & 1] for i in range(8)], dtype=float)


def _kuhn_tets() -> np.ndarray:
    tets = []
    for perm in permutations(range(3)):
        v = np.zeros(3)
        ids = [0]
        for ax in perm:
            v = v.copy()
            v[ax] = 1.0
            ids.append(int(v[0]) + 2 * int(v[1]) + 4 * int(v[2]))
        tets.append(ids)
    return np.array(tets, dtype=np.int64)


KUHN = _kuhn_tets()  # (6, 4) corner ids


def _edge_point(pa, pb, fa, fb):
    t = fa / (fa - fb)
    return pa + t * (pb - pa)


def clip_tet(P: np.ndarray, f: np.ndarray):
    """Clip tetrahedron ``P`` (4,3) with vertex values ``f`` by ``f >= 0``.

    Returns (list of fluid tetrahedra as (4,3) arrays, list of zero-set
    triangles as (3,3) arrays).
    """
    pos = [i for i in range(4) if f[i] >= 0.0]
    neg = [i for i in range(4) if f[i] < 0.0]
    if len(neg) == 0:
        return [P], []
    if len(pos) == 0:
        return [], []
    if len(pos) == 1:
        a = pos[0]
        q = [_edge_point(P[a], P[j], f[a], f[j]) for j in neg]
        return [np.array([P[a], q[0], q[1], q[2]])], [np.array(q)]
    if len(pos) == 3:
        d = neg[0]
        A = [P[i] for i in pos]
        B = [_edge_point(P[i], P[d], f[i], f[d]) for i in pos]
        return _prism(A, B), [np.array(B)]
    a, b = pos
    c, d = neg
    A = [P[a], _edge_point(P[a], P[c], f[a], f[c]), _edge_point(P[a], P[d], f[a], f[d])]
    B = [P[b], _edge_point(P[b], P[c], f[b], f[c]), _edge_point(P[b], P[d], f[b], f[d])]
    quad = [A[1], A[2], B[2], B[1]]
    return _prism(A, B), [np.array([quad[0], quad[1], quad[2]]), np.array([quad[0], quad[2], quad[3]])]


def _prism(A, B):
    return [
        np.array([A[0], A[1], A[2], B[0]]),
        np.array([A[1], A[2], B[0], B[1]]),
        np.array([A[2], B[0], B[1], B[2]]),
    ]


def clip_triangle(P: np.ndarray, f: np.ndarray):
    """Clip triangle ``P`` (3,3) by ``f >= 0``; returns a list of triangles."""
    poly = []
    for k in range(3):
        i, j = k, (k + 1) % 3
        if f[i] >= 0.0:
            poly.append(P[i])
        if (f[i] >= 0.0) != (f[j] >= 0.0):
            poly.append(_edge_point(P[i], P[j], f[i], f[j]))
    if len(poly) < 3:
        return []
    return [np.array([poly[0], poly[k], poly[k + 1]]) for k in range(1, len(poly) - 1)]


@dataclass
class CellQuadrature:
    """Quadrature for one cut cell: volume points/weights and boundary
    points/weights/outward normals (Dirichlet boundary: cut surface and the
    box faces inside this cell)."""

    xv: np.ndarray  # (mv, 3)
    wv: np.ndarray  # (mv,)
    xs: np.ndarray  # (ms, 3)
    ws: np.ndarray  # (ms,)
    ns: np.ndarray  # (ms, 3)
    volume: float


def cut_cell_quadrature(
    phi,
    lo: np.ndarray,
    h: float,
    q: int,
    subdiv: int = 1,
    box_faces: bool = True,
    cell_faces: bool = False,
) -> CellQuadrature:
    """Quadrature of ``{phi_lin >= 0}`` in the cell ``[lo, lo+h]^3``.

    ``box_faces`` adds the parts of the unit-box faces inside the cell to the
    boundary rule; ``cell_faces`` adds every face of the cell instead (used to
    check the per-cell Green identity).
    """
    tq, tw = tet_rule(q)
    rq, rw = tri_rule(q)
    hs = h / subdiv
    xv, wv, xs, ws, ns = [], [], [], [], []
    vol = 0.0
    for sz in range(subdiv):
        for sy in range(subdiv):
            for sx in range(subdiv):
                base = lo + hs * np.array([sx, sy, sz], dtype=float)
                C = base[None, :] + hs * _CUBE_CORNERS
                fc = phi(C[:, 0], C[:, 1], C[:, 2])
                if np.all(fc < 0.0):
                    continue
                for tet in KUHN:
                    P = C[tet]
                    f = fc[tet]
                    pieces, surf = clip_tet(P, f)
                    for T in pieces:
                        J = np.stack([T[1] - T[0], T[2] - T[0], T[3] - T[0]], axis=1)
                        det = abs(float(np.linalg.det(J)))
                        if det <= 0.0:
                            continue
                        xv.append(T[0][None, :] + tq @ J.T)
                        wv.append(det * tw)
                        vol += det / 6.0
                    if surf:
                        # gradient of the linear interpolant on this tet
                        J = np.stack([P[1] - P[0], P[2] - P[0], P[3] - P[0]], axis=0)
                        g = np.linalg.solve(J, f[1:] - f[0])
                        gn = np.linalg.norm(g)
                        if gn > 0.0:
                            nrm = -g / gn
                            for S in surf:
                                cr = np.cross(S[1] - S[0], S[2] - S[0])
                                area2 = float(np.linalg.norm(cr))
                                if area2 <= 0.0:
                                    continue
                                E2 = np.stack([S[1] - S[0], S[2] - S[0]], axis=1)
                                xs.append(S[0][None, :] + rq @ E2.T)
                                ws.append(area2 * rw)
                                ns.append(np.broadcast_to(nrm, (rq.shape[0], 3)))
                    if box_faces or cell_faces:
                        for face in ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)):
                            F = P[list(face)]
                            for ax in range(3):
                                planes = (
                                    ((-1.0, lo[ax]), (1.0, lo[ax] + h))
                                    if cell_faces
                                    else ((-1.0, 0.0), (1.0, 1.0))
                                )
                                for side, val in planes:
                                    if np.all(np.abs(F[:, ax] - val) <= 1e-14):
                                        for S in clip_triangle(F, f[list(face)]):
                                            cr = np.cross(S[1] - S[0], S[2] - S[0])
                                            area2 = float(np.linalg.norm(cr))
                                            if area2 <= 0.0:
                                                continue
                                            E2 = np.stack([S[1] - S[0], S[2] - S[0]], axis=1)
                                            nrm = np.zeros(3)
                                            nrm[ax] = side
                                            xs.append(S[0][None, :] + rq @ E2.T)
                                            ws.append(area2 * rw)
                                            ns.append(np.broadcast_to(nrm, (rq.shape[0], 3)))
    cat = lambda L, shape: np.concatenate(L) if L else np.zeros(shape)
    return CellQuadrature(
        cat(xv, (0, 3)), cat(wv, (0,)), cat(xs, (0, 3)), cat(ws, (0,)), cat(ns, (0, 3)), vol
    )
