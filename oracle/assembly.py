"""Global assembly oracle (CPU) -- test infrastructure only.

Rebuilds the full-space operator of a ``CutCellProblem`` the way the
reference assembles its 3D systems: per element, explicit Kronecker blocks of
1D interval forms (``AxisForms.interval`` + ``_kron3_block``,
code/bell_3d_core.py:172-232, 338-390) accumulated as COO triplets, then CSR
and symmetrised (code/bell_3d_core.py:392-399).  The 1D forms are recomputed
here with SciPy B-splines and Gauss-Legendre quadrature of order
max(5, p+3) (code/bell_3d_core.py:288), independently of the product's
Cox-de Boor tables; weak-penalty box faces follow code/cut_3d_sbp.py:426-460.
Cut elements contribute the problem's dense cut blocks unchanged (their
quadrature is checked separately by geometric identities).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.interpolate import BSpline

from .aggregation import open_uniform_knots


def interval_forms(n: int, p: int, q: int | None = None):
    """Per-element 1D mass and stiffness (n, p+1, p+1)."""
    q = q or max(5, p + 3)
    t = open_uniform_knots(n, p)
    g, w = np.polynomial.legendre.leggauss(q)
    h = 1.0 / n
    M = np.zeros((n, p + 1, p + 1))
    K = np.zeros((n, p + 1, p + 1))
    for e in range(n):
        a, b = e * h, (e + 1) * h
        x = 0.5 * (b - a) * g + 0.5 * (b + a)
        wq = 0.5 * (b - a) * w
        V = np.zeros((p + 1, q))
        D = np.zeros((p + 1, q))
        for i in range(p + 1):
            c = np.zeros(n + p)
            c[e + i] = 1.0
            s = BSpline(t, c, p, extrapolate=False)
            V[i] = np.nan_to_num(s(x))
            D[i] = np.nan_to_num(s.derivative()(x))
        M[e] = (V * wq) @ V.T
        K[e] = (D * wq) @ D.T
    return M, K


def face_forms(n: int, p: int, beta: float):
    """Weak-penalty factor beta t t^T - s (t dt^T + dt t^T) on the first and last element."""
    t = open_uniform_knots(n, p)
    out = []
    for e, x, s in ((0, 0.0, -1.0), (n - 1, 1.0, 1.0)):
        tr = np.zeros(p + 1)
        dt = np.zeros(p + 1)
        for i in range(p + 1):
            c = np.zeros(n + p)
            c[e + i] = 1.0
            sp_ = BSpline(t, c, p)
            tr[i] = sp_(x)
            dt[i] = sp_.derivative()(x)
        out.append(beta * np.outer(tr, tr) - s * (np.outer(tr, dt) + np.outer(dt, tr)))
    return out


def assemble_full(prob) -> sp.csr_matrix:
    n, p = prob.n_elements, prob.degree
    p1 = p + 1
    nb = n + p
    M, K = interval_forms(n, p)
    Kt = [prob.a_stiff * K.copy() for _ in range(3)]
    if prob.nitsche:
        lo, hi = face_forms(n, p, prob.beta)
        for ax in range(3):
            Kt[ax][0] = Kt[ax][0] + lo
            Kt[ax][n - 1] = Kt[ax][n - 1] + hi
    rows_l, cols_l, vals_l = [], [], []
    et = prob.elem_type
    cut_index = {int(c): k for k, c in enumerate(prob.cut_ids)}
    for ez in range(n):
        for ey in range(n):
            for ex in range(n):
                typ = et[ez, ey, ex]
                if typ == 0:
                    continue
                gx = np.arange(ex, ex + p1)
                gy = np.arange(ey, ey + p1)
                gz = np.arange(ez, ez + p1)
                rows = ((gz[:, None] * nb + gy[None, :])[:, :, None] * nb + gx[None, None, :]).reshape(-1)
                if typ == 1:
                    B = (
                        np.kron(np.kron(M[ez], M[ey]), prob.a_mass * M[ex] + Kt[0][ex])
                        + np.kron(np.kron(M[ez], Kt[1][ey]), M[ex])
                        + np.kron(np.kron(Kt[2][ez], M[ey]), M[ex])
                    )
                else:
                    B = prob.cut_mats[cut_index[(ez * n + ey) * n + ex]]
                rows_l.append(np.repeat(rows, rows.size))
                cols_l.append(np.tile(rows, rows.size))
                vals_l.append(B.reshape(-1))
    N = nb**3
    A = sp.coo_matrix((np.concatenate(vals_l), (np.concatenate(rows_l), np.concatenate(cols_l))), shape=(N, N)).tocsr()
    return ((A + A.T) * 0.5).tocsr()
