"""Aggregation oracle (CPU) -- test infrastructure only.

Restates, one small coordinate at a time:
* ``polynomial_coefficients`` (code/cut_spline_sbp.py:148-153) with SciPy
  B-splines (the reference's evaluator);
* ``_greville_3d`` / ``_monomial_rows_3d`` (code/bell_3d_core.py:435-458);
* ``polynomial_preserving_extension_3d`` (code/bell_3d_core.py:471-542):
  interior = gamma >= 0.04, nearest interior Greville neighbours, stencil
  n_terms+8 growing by 8 while matrix_rank(tol=1e-10) < n_terms (at most
  6 n_terms), lstsq weights, |w| > 1e-14 kept;
* ``restrict_spd`` (code/bell_3d_core.py:550-552): 1/2 (E^T A E + (E^T A E)^T).
"""

from __future__ import annotations

import numpy as np
import scipy.sparse as sp
from scipy.interpolate import BSpline


def open_uniform_knots(n: int, p: int) -> np.ndarray:
    """code/cut_spline_sbp.py:57-65."""
    h = 1.0 / n
    return np.concatenate([np.zeros(p + 1), np.arange(1, n, dtype=float) * h, np.ones(p + 1)])


def greville(n: int, p: int) -> np.ndarray:
    t = open_uniform_knots(n, p)
    return np.array([np.sum(t[i + 1 : i + p + 1]) / p for i in range(n + p)])


def basis_matrix(n: int, p: int, x: np.ndarray) -> np.ndarray:
    t = open_uniform_knots(n, p)
    nb = n + p
    V = np.zeros((nb, x.size))
    for i in range(nb):
        c = np.zeros(nb)
        c[i] = 1.0
        V[i] = np.nan_to_num(BSpline(t, c, p, extrapolate=False)(x), nan=0.0)
    return V


def polynomial_coefficients(n: int, p: int, max_degree: int) -> np.ndarray:
    g = greville(n, p)
    A = basis_matrix(n, p, g).T
    return np.asarray([np.linalg.solve(A, g**r) for r in range(max_degree + 1)])


def greville_3d(n: int, p: int) -> np.ndarray:
    g = greville(n, p)
    nb = n + p
    return np.column_stack([np.tile(np.tile(g, nb), nb), np.tile(np.repeat(g, nb), nb), np.repeat(g, nb * nb)])


def monomial_rows_3d(n: int, p: int, degree: int) -> np.ndarray:
    c = polynomial_coefficients(n, p, degree)
    rows = []
    for total in range(degree + 1):
        for a in range(total + 1):
            for b in range(total - a + 1):
                cc = total - a - b
                rows.append(np.einsum("k,j,i->kji", c[cc], c[b], c[a]).reshape(-1))
    return np.vstack(rows)


def extension_3d(gamma: np.ndarray, n: int, p: int, support_threshold: float = 0.04):
    gamma = np.asarray(gamma, dtype=float)
    active = np.where(gamma > 0.0)[0]
    interior = np.where(gamma >= support_threshold)[0]
    small = np.array([i for i in active if gamma[i] < support_threshold], dtype=int)
    poly = monomial_rows_3d(n, p, p)
    n_terms = poly.shape[0]
    G = greville_3d(n, p)
    col = {int(g): j for j, g in enumerate(interior)}
    rows_t, cols_t, vals_t = [], [], []
    for g in interior:
        rows_t.append(int(g))
        cols_t.append(col[int(g)])
        vals_t.append(1.0)
    for b in small:
        dist = np.linalg.norm(G[interior] - G[int(b)][None, :], axis=1)
        ordered = interior[np.argsort(dist[None, :], axis=1)[0]]
        k = n_terms
        chosen = ordered[: k + 8]
        C = poly[:, chosen]
        while np.linalg.matrix_rank(C, tol=1.0e-10) < n_terms and len(chosen) < min(len(ordered), 6 * n_terms):
            k += 8
            chosen = ordered[: k + 8]
            C = poly[:, chosen]
        w, *_ = np.linalg.lstsq(C, poly[:, int(b)], rcond=None)
        for g, wt in zip(chosen, w):
            if abs(wt) > 1.0e-14:
                rows_t.append(int(b))
                cols_t.append(col[int(g)])
                vals_t.append(float(wt))
    E = sp.csr_matrix((vals_t, (rows_t, cols_t)), shape=(gamma.size, interior.size))
    E.sort_indices()
    return E, interior, small


def restrict_spd(A, E):
    B = (E.T @ A @ E).tocsr()
    return ((B + B.T) * 0.5).tocsr()
