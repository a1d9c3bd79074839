"""Open-uniform maximal-smoothness B-spline bases on [0, 1] (host setup).

The basis matches ``make_open_uniform_basis`` (code/cut_spline_sbp.py:52-76):
knots ``[0]*(p+1) + [h, 2h, ..., (n-1)h] + [1]*(p+1)``, ``n+p`` functions,
Greville abscissae ``sum(t[i+1:i+p+1])/p``.  On element ``e`` the nonzero
functions are ``e .. e+p`` (code/cut_assembly.py:71-78).  Values come from the
Cox-de Boor recursion (Piegl & Tiller, The NURBS Book, algorithm A2.2) and
first derivatives from the degree-lowering identity
``N'_{i,p} = p (N_{i,p-1}/(t_{i+p}-t_i) - N_{i+1,p-1}/(t_{i+p+1}-t_{i+1}))``,
the same identity code/cut_assembly.py:56-66 uses.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class OpenUniformBasis:
    n_elements: int
    degree: int
    knots: np.ndarray
    greville: np.ndarray

    @property
    def n_basis(self) -> int:
        return self.n_elements + self.degree

    @property
    def h(self) -> float:
        return 1.0 / self.n_elements


def make_basis(n_elements: int, degree: int) -> OpenUniformBasis:
    if n_elements < 1:
        raise ValueError("n_elements must be at least 1")
    if degree < 1:
        raise ValueError("degree must be at least 1")
    h = 1.0 / n_elements
    knots = np.concatenate(
        [np.zeros(degree + 1), np.arange(1, n_elements, dtype=float) * h, np.ones(degree + 1)]
    )
    nb = n_elements + degree
    greville = np.array([np.sum(knots[i + 1 : i + degree + 1]) / degree for i in range(nb)])
    return OpenUniformBasis(int(n_elements), int(degree), knots, greville)


def element_of(basis: OpenUniformBasis, x: np.ndarray) -> np.ndarray:
    """Element index containing each point (the right end belongs to the last element)."""
    e = np.floor(np.asarray(x, dtype=float) * basis.n_elements).astype(np.int64)
    return np.clip(e, 0, basis.n_elements - 1)


def _cox_de_boor(t: np.ndarray, span: np.ndarray, x: np.ndarray, deg: int) -> np.ndarray:
    """Nonzero degree-``deg`` functions ``span-deg .. span`` at ``x``; shape (m, deg+1)."""
    m = x.shape[0]
    N = np.zeros((m, deg + 1))
    N[:, 0] = 1.0
    left = np.zeros((m, deg + 1))
    right = np.zeros((m, deg + 1))
    for j in range(1, deg + 1):
        left[:, j] = x - t[span + 1 - j]
        right[:, j] = t[span + j] - x
        saved = np.zeros(m)
        for r in range(j):
            den = right[:, r + 1] + left[:, j - r]
            temp = N[:, r] / den
            N[:, r] = saved + right[:, r + 1] * temp
            saved = left[:, j - r] * temp
        N[:, j] = saved
    return N


def local_values(basis: OpenUniformBasis, elem: np.ndarray, x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Values and first derivatives of the ``p+1`` functions living on ``elem``.

    ``elem`` and ``x`` are broadcast 1-D arrays of equal length; the points may
    lie on the element's closed interval.  Returns two arrays of shape
    ``(m, p+1)``; column ``i`` belongs to global function ``elem + i``.
    """
    p = basis.degree
    t = basis.knots
    x = np.asarray(x, dtype=float).ravel()
    elem = np.broadcast_to(np.asarray(elem, dtype=np.int64), x.shape).ravel()
    span = elem + p
    N = _cox_de_boor(t, span, x, p)
    low = _cox_de_boor(t, span, x, p - 1)  # functions span-p+1 .. span of degree p-1
    D = np.zeros_like(N)
    for i in range(p + 1):
        g = span - p + i
        if i >= 1:
            den = t[g + p] - t[g]
            D[:, i] += np.where(den > 0, p * low[:, i - 1] / np.where(den > 0, den, 1.0), 0.0)
        if i <= p - 1:
            den = t[g + p + 1] - t[g + 1]
            D[:, i] -= np.where(den > 0, p * low[:, i] / np.where(den > 0, den, 1.0), 0.0)
    return N, D


def global_values(basis: OpenUniformBasis, x: np.ndarray) -> np.ndarray:
    """Dense (m, n_basis) table of basis values (setup-sized inputs only)."""
    x = np.asarray(x, dtype=float).ravel()
    e = element_of(basis, x)
    N, _ = local_values(basis, e, x)
    out = np.zeros((x.size, basis.n_basis))
    for i in range(basis.degree + 1):
        out[np.arange(x.size), e + i] = N[:, i]
    return out


def gauss_legendre01(q: int) -> tuple[np.ndarray, np.ndarray]:
    g, w = np.polynomial.legendre.leggauss(q)
    return 0.5 * (g + 1.0), 0.5 * w


def element_matrices_1d(basis: OpenUniformBasis, q: int | None = None):
    """Full-element 1D mass and stiffness blocks, shape (n_elements, p+1, p+1).

    These are the per-axis factors of every uncut 3D element block, as in
    ``AxisForms.interval`` (code/bell_3d_core.py:172-200).
    """
    p = basis.degree
    q = q or (p + 2)
    xg, wg = gauss_legendre01(q)
    ne = basis.n_elements
    h = basis.h
    e = np.repeat(np.arange(ne), q)
    x = (e + np.tile(xg, ne)) * h
    w = np.tile(wg, ne) * h
    N, D = local_values(basis, e, x)
    N = N.reshape(ne, q, p + 1)
    D = D.reshape(ne, q, p + 1)
    w = w.reshape(ne, q)
    M = np.einsum("eqi,eq,eqj->eij", N, w, N)
    K = np.einsum("eqi,eq,eqj->eij", D, w, D)
    return M, K


def polynomial_coefficients(basis: OpenUniformBasis, max_degree: int) -> np.ndarray:
    """Spline coefficients of the monomials ``x^r`` (r <= max_degree) by Greville
    interpolation, as ``polynomial_coefficients`` (code/cut_spline_sbp.py:148-153)."""
    A = global_values(basis, basis.greville)
    return np.asarray([np.linalg.solve(A, basis.greville**r) for r in range(max_degree + 1)])
