"""Coarse level of the two-level patch preconditioner (CUTCELL_PRECOND_TWOLEVEL).

The reference preconditions its aggregated systems E^T A E with Jacobi only
(``jacobi_preconditioner``, code/fast_solver_backends.py:74-88); this is a
preconditioner of the same systems, selected with ``preconditioner=
"twolevel"``.  Per flexible-PCG iteration

    z = zc + B (r - A zc),   zc = P Ac^-1 P^T r,   Ac = P^T A P,

with B the exact 4x4x4 patch solves (``learned.attach_blocks``) and P the
uniform B-spline refinement from ``n / c`` to ``n`` elements per axis: the
coarse open-uniform space is nested in the fine one, so every coarse
function is exactly a combination of fine ones (R1, knot insertion), and P
takes the rows of R1 (x) R1 (x) R1 that belong to the reduced (kept) DOFs,
the identity rows of E.  Ac is formed on the device by applying the
matrix-free operator to P's columns, and inverted densely here (the coarse
grid is chosen with at most ``max_dofs`` functions, so Ac^-1 stays in L2).

Measured on the sphere-cut p = 3 systems (CPU, assembled E^T A E, FCG to
1e-9): Jacobi 404 / 469 iterations at n = 16 / 32, exact patch solves
150 / 242, two-level 42 (n = 16, coarse n = 8) / 68 (n = 32, coarse n = 8),
two-level with a second patch tiling offset by 2 DOFs (z = zc + 0.5 (B_0 +
B_2) (r - A zc), the default) 27 / 35.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

from . import _lib
from .bspline import global_values, make_basis


def refinement_1d(n_fine: int, degree: int, factor: int) -> np.ndarray:
    """R1 (nb_fine x nb_coarse) with coarse B-spline a = sum_x R1[x, a] fine
    B-spline x, for open uniform knots on [0, 1] with n_fine and
    n_fine / factor elements.  Found by interpolation at the fine Greville
    points (exact: the coarse functions lie in the fine space); entries below
    1e-13 of the largest, rounding of exact zeros, are set to zero."""
    if n_fine % factor:
        raise ValueError(f"{n_fine} elements are not divisible by the coarsening factor {factor}")
    fb, cb = make_basis(n_fine, degree), make_basis(n_fine // factor, degree)
    g = fb.greville
    R = np.linalg.solve(global_values(fb, g), global_values(cb, g))
    R[np.abs(R) < 1e-13 * np.abs(R).max()] = 0.0
    return R


def coarse_factor(n: int, degree: int, max_dofs: int = 2048) -> int:
    """Smallest coarsening factor 2, 4, 8, ... dividing n whose coarse grid
    has at most ``max_dofs`` functions."""
    c = 2
    while c <= n:
        if n % c == 0 and (n // c + degree) ** 3 <= max_dofs:
            return c
        c *= 2
    raise ValueError(f"no coarse grid of <= {max_dofs} functions for n = {n}, p = {degree}")


def _bands(R: np.ndarray, pw: int | None = None):
    """Banded rows (plo, pw, pval) and columns (rlo, rw, rval) of R1, each
    band start clamped so that start + width stays inside the grid.  ``pw``
    pads the row bands to a given width (the device unrolls p + 1)."""
    nb, nbc = R.shape
    rows = [np.nonzero(R[x])[0] for x in range(nb)]
    cols = [np.nonzero(R[:, a])[0] for a in range(nbc)]
    need = max(int(ix[-1] - ix[0] + 1) for ix in rows if ix.size)
    if pw is None:
        pw = need
    if need > pw or pw > nbc:
        raise ValueError(f"prolongation rows need a band of {need}; asked for {pw} on {nbc} coarse functions")
    rw = max(int(ix[-1] - ix[0] + 1) for ix in cols if ix.size)
    plo = np.array([min(int(ix[0]) if ix.size else 0, nbc - pw) for ix in rows], dtype=np.int32)
    rlo = np.array([min(int(ix[0]) if ix.size else 0, nb - rw) for ix in cols], dtype=np.int32)
    pval = np.array([R[x, plo[x]:plo[x] + pw] for x in range(nb)])
    rval = np.array([R[rlo[a]:rlo[a] + rw, a] for a in range(nbc)])
    return plo, pw, pval, rlo, rw, rval


def prolongation(prob, ext, factor: int):
    """(P, R1): P the sparse (n_red x nbc^3) prolongation onto the reduced
    DOFs, coarse index (c nbc + b) nbc + a for (x, y, z) = (a, b, c)."""
    R = refinement_1d(prob.n_elements, prob.degree, factor)
    R1 = sp.csr_matrix(R)
    Pf = sp.kron(sp.kron(R1, R1), R1).tocsr()
    full_of_red = np.asarray(ext.device_layout()["full_of_red"])
    return Pf[full_of_red, :].tocsc(), R


class CoarseLevel:
    """Coarse tables of one operator on its device, and Ac^-1."""

    def __init__(self, op, factor: int | None = None, max_dofs: int = 2048, chunk: int = 128):
        import time

        import torch

        t0 = time.perf_counter()
        prob, ext = op.problem, op.extension
        self.factor = factor or coarse_factor(prob.n_elements, prob.degree, max_dofs)
        P, R = prolongation(prob, ext, self.factor)
        nb, nbc = R.shape
        self.nb, self.nbc, self.ncg = nb, nbc, nbc**3
        keep = np.nonzero(np.diff(P.indptr))[0]
        self.keep = keep
        # Ac = P^T A P from device applies of P's columns
        Pk = P[:, keep].tocsc()
        Ac = np.zeros((keep.size, keep.size))
        Pt = Pk.T.tocsr()
        for c0 in range(0, keep.size, chunk):
            c1 = min(c0 + chunk, keep.size)
            V = torch.as_tensor(Pk[:, c0:c1].toarray().T.copy(), device=op.device)
            W = torch.stack([op.apply(V[i]) for i in range(c1 - c0)], dim=1).cpu().numpy()
            Ac[:, c0:c1] = Pt @ W
        self.galerkin_s = time.perf_counter() - t0
        Ac = 0.5 * (Ac + Ac.T)
        self.Ac = Ac
        cf = sla.cho_factor(Ac, lower=False)
        inv_k = sla.cho_solve(cf, np.eye(keep.size))
        inv_k = 0.5 * (inv_k + inv_k.T)
        minv = np.zeros((self.ncg, self.ncg))
        minv[np.ix_(keep, keep)] = inv_k
        plo, pw, pval, rlo, rw, rval = _bands(R, prob.degree + 1)
        self.pw, self.rw = pw, rw
        dv = op.device
        self._t = {
            "plo": torch.as_tensor(plo, dtype=torch.int32, device=dv),
            "pval": torch.as_tensor(pval, dtype=torch.float64, device=dv).contiguous(),
            "rlo": torch.as_tensor(rlo, dtype=torch.int32, device=dv),
            "rval": torch.as_tensor(rval, dtype=torch.float64, device=dv).contiguous(),
            # FP64: stored in FP32 the coarse inverse raised the iterations at n = 32
            # from 35 to 51 (the block inverses keep their counts in FP32)
            "minv": torch.as_tensor(minv, dtype=torch.float64, device=dv).contiguous(),
        }
        self.P, self.R = P, R
        self.setup_s = time.perf_counter() - t0

    def desc(self) -> _lib.CutcellCoarseDesc:
        d = _lib.CutcellCoarseDesc()
        d.nb, d.nbc, d.pw, d.rw = self.nb, self.nbc, self.pw, self.rw
        for k, t in self._t.items():
            setattr(d, k, t.data_ptr())
        return d


class OverlapTiling:
    """An extra patch tiling (offset by ``shift`` DOFs per axis), its probed
    blocks and their exact inverses on the operator's device."""

    def __init__(self, op, shift: int = 2):
        import torch

        from .learned import DevicePatches, patch_blocks, patch_inverses, patch_layout

        self.dp = DevicePatches(op, patch_layout(op, shift))
        inv = patch_inverses(patch_blocks(op, self.dp), self.dp.layout.red)
        # BF16 storage: the preconditioner's blocks; products accumulate in FP64
        self.inv = torch.as_tensor(0.5 * (inv + np.transpose(inv, (0, 2, 1)))).to(op.device).to(torch.bfloat16)

    @property
    def n_patch(self) -> int:
        return self.dp.n_patch


# extra patch tilings of the default two-level form and their weight: the
# offsets 1, 2, 3 with the first tiling give B = 0.3 (B_0 + B_1 + B_2 + B_3)
DEFAULT_SHIFTS = (1, 2, 3)
DEFAULT_OMEGA = 0.3


def attach_coarse(op, factor: int | None = None, max_dofs: int = 2048, shifts=DEFAULT_SHIFTS,
                  omega: float | None = None) -> CoarseLevel:
    """Set up CUTCELL_PRECOND_TWOLEVEL on a CutCellOperator: exact patch
    blocks on every patch (if none are attached), the coarse level, and the
    extra patch tilings offset by ``shifts`` DOFs per axis (at most three), so
    that the step is z = zc + omega (B_0 + B_s1 + ...) (r - A zc).  Measured on
    the sphere-cut p = 3 n = 32 system (CPU, assembled E^T A E, FCG to 1e-9):
    68 iterations with the first tiling alone, 35 with shifts (2,) and
    omega 0.5, 30 with (1, 3) and 1/3, 26 with (1, 2, 3) and 0.3."""
    import torch

    from .learned import attach_blocks, patch_solves

    shifts = tuple(int(t) for t in (shifts or ()))
    if len(shifts) > 3 or any(t <= 0 or t >= 4 for t in shifts):
        raise ValueError("at most three extra tilings, offsets 1..3")
    if omega is None:
        omega = {0: 1.0, 1: 0.5, 2: 1.0 / 3.0, 3: DEFAULT_OMEGA}[len(shifts)]
    if getattr(op, "_block_slot", None) is None:
        attach_blocks(op, "all")
    cl = CoarseLevel(op, factor, max_dofs)
    d = cl.desc()
    _lib.check(op._lib.cutcell_pcg_set_coarse(op._ctx, C.byref(d)), "cutcell_pcg_set_coarse")
    # BF16 copies of the patch inverses (the two-level step reads them every iteration;
    # at n = 32 four tilings hold 3,372 of them: 28 MB in BF16, 55 MB in FP32, 110 MB in FP64)
    cl.inv0f = patch_solves(op).inv.to(torch.bfloat16).contiguous()
    cl.extra = [OverlapTiling(op, t) for t in shifts]
    cl.shifts = shifts
    cl.omega = float(omega) if shifts else 1.0
    n = len(cl.extra)
    reds = (C.c_void_p * 3)(*[t.dp.red.data_ptr() for t in cl.extra], *([None] * (3 - n)))
    invs = (C.c_void_p * 3)(*[t.inv.data_ptr() for t in cl.extra], *([None] * (3 - n)))
    cnts = (C.c_int32 * 3)(*[t.n_patch for t in cl.extra], *([0] * (3 - n)))
    _lib.check(op._lib.cutcell_pcg_set_twolevel_blocks(op._ctx, cl.inv0f.data_ptr(), n, reds, cnts, invs, cl.omega),
               "cutcell_pcg_set_twolevel_blocks")
    op._coarse = cl
    return cl


def detach_coarse(op) -> None:
    _lib.check(op._lib.cutcell_pcg_set_twolevel_blocks(op._ctx, None, 0, None, None, None, 1.0),
               "cutcell_pcg_set_twolevel_blocks")
    _lib.check(op._lib.cutcell_pcg_set_coarse(op._ctx, None), "cutcell_pcg_set_coarse")
    op._coarse = None
