"""Jacobi-PCG oracle (CPU, FP64) -- test infrastructure only.

* ``solve_cpu_cg`` restates code/fast_solver_backends.py:90-132: SciPy ``cg``
  with ``rtol=tol, atol=0``, a Jacobi ``LinearOperator`` whose inverse is zero
  on zero diagonal entries (code/fast_solver_backends.py:74-87), iterations
  counted by callback, success iff ``info == 0`` and the true residual
  ``||Ax-b||/||b||`` is at most ``max(10 tol, 1e-14)``.
* ``cg_loop`` restates the hand-written loop of solve_gpu_cg
  (code/fast_solver_backends.py:236-289) in NumPy: the iteration counted is
  the one in which ``||r||/||b|| <= tol`` first holds, breakdown on
  ``p.Ap <= 0``, ``z = r`` where the diagonal is zero.
"""

from __future__ import annotations

from time import perf_counter

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla


def as_csr(A):
    return A.tocsr() if sp.issparse(A) else sp.csr_matrix(np.asarray(A, dtype=float))


def relative_residual(A, x, b) -> float:
    """code/fast_solver_backends.py:63-71."""
    A = as_csr(A)
    b = np.asarray(b, dtype=float)
    den = float(np.linalg.norm(b))
    if den == 0.0:
        den = 1.0
    return float(np.linalg.norm(A @ x - b) / den)


def jacobi_inverse(A) -> np.ndarray:
    d = as_csr(A).diagonal().astype(float)
    inv = np.zeros_like(d)
    m = np.abs(d) > 0.0
    inv[m] = 1.0 / d[m]
    return inv


def solve_cpu_cg(A, b, *, tol=1e-8, maxiter=5000, preconditioner="jacobi"):
    A = as_csr(A)
    b = np.asarray(b, dtype=float)
    count = 0

    def cb(_):
        nonlocal count
        count += 1

    M = None
    if preconditioner == "jacobi":
        inv = jacobi_inverse(A)
        M = spla.LinearOperator(A.shape, matvec=lambda v: inv * v, dtype=float)
    tic = perf_counter()
    x, info = spla.cg(A, b, rtol=tol, atol=0.0, maxiter=maxiter, M=M, callback=cb)
    elapsed = perf_counter() - tic
    rel = relative_residual(A, x, b)
    success = bool(info == 0 and np.isfinite(rel) and rel <= max(10.0 * tol, 1e-14))
    return x, {
        "success": success,
        "iterations": int(count if count else max(info, 0)),
        "elapsed_s": elapsed,
        "relative_residual": rel,
        "info": int(info),
    }


def cg_loop(A, b, *, tol=1e-8, maxiter=5000, preconditioner="jacobi"):
    A = as_csr(A)
    b = np.asarray(b, dtype=float)
    x = np.zeros_like(b)
    r = b - A @ x
    d = A.diagonal()
    pre = preconditioner == "jacobi"

    def Minv(v):
        if not pre:
            return v.copy()
        return np.where(np.abs(d) > 0.0, v / np.where(np.abs(d) > 0.0, d, 1.0), v)

    z = Minv(r)
    p = z.copy()
    rz = float(r @ z)
    bn = float(np.linalg.norm(b))
    if bn == 0.0:
        bn = 1.0
    status, it = "maximum iterations reached", 0
    for k in range(1, maxiter + 1):
        Ap = A @ p
        pap = float(p @ Ap)
        if pap <= 0.0 or not np.isfinite(pap):
            status, it = "CG breakdown: non-positive curvature", k
            break
        alpha = rz / pap
        x = x + alpha * p
        r = r - alpha * Ap
        it = k
        if np.linalg.norm(r) / bn <= tol:
            status = "converged"
            break
        z = Minv(r)
        rzn = float(r @ z)
        p = z + (rzn / rz) * p
        rz = rzn
    rel = relative_residual(A, x, b)
    return x, {
        "message": status,
        "iterations": it,
        "relative_residual": rel,
        "success": status == "converged" and rel <= max(10.0 * tol, 1e-14),
    }
