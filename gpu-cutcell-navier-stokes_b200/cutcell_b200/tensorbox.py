"""Tensor-product cut boxes: the Kronecker SBP forms and the 3D cut-box
Poisson solve of code/cut_3d_sbp.py, with the matrix-free device operator.

The cut box is ``[a_x, 1] x [a_y, 1] x [a_z, 1]`` with ``a_i = h * frac_i``.
Every form the reference assembles (code/cut_3d_sbp.py:89-146) is a sum of
Kronecker products of 1D cut-interval forms, and so is the extension
``E = Ez (x) Ey (x) Ex``; the pullback therefore factors per axis:

    E^T (Cz (x) Cy (x) Cx) E = (Ez^T Cz Ez) (x) (Ey^T Cy Ey) (x) (Ex^T Cx Ex).

The device never forms the N x N matrices: ``KronOperator`` holds the reduced
1D factors (n_a x n_a per axis and form, a few KB) and applies

    H  = Hz (x) Hy (x) Hx
    K  = Hz (x) Hy (x) Kx + Hz (x) Ky (x) Hx + Kz (x) Hy (x) Hx
    Qx = Hz (x) Hy (x) Qx,  Qy = Hz (x) Qy (x) Hx,  Qz = Qz (x) Hy (x) Hx
    Sx, Sy, Sz likewise with the boundary forms
    A  = Hz (x) Hy (x) Ax + Hz (x) Ay (x) Hx + Az (x) Hy (x) Hx

by three sum-factorised passes (x, y, z), where ``A_a = K_a + beta F_a - N_a -
N_a^T`` is the per-axis weak-penalty Poisson factor of solve_poisson_3d
(code/cut_3d_sbp.py:386-503): F_a the face-trace mass ``tL tL^T + tR tR^T``
and N_a the trace / normal-derivative form ``-tL dL^T + tR dR^T``.

``solve_poisson_3d`` restates the reference wrapper with an opt-in
``linear_solver=``: ``None`` keeps its dense ``np.linalg.solve``, ``"b200"``
solves the same system matrix-free on the device through ``solve_spd``, and
a callable ``(A, b) -> x`` receives the assembled matrix (the routing a
maintainer adds at code/cut_3d_sbp.py:503).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from math import pi

import numpy as np

from . import _lib
from .aggregation import extension_1d
from .bspline import OpenUniformBasis, element_of, local_values, make_basis

# form selectors of cutcell_apply_form (include/cutcell_b200.h)
FORMS = {"A": 0, "H": 1, "K": 2, "Qx": 3, "Qy": 4, "Qz": 5, "Sx": 6, "Sy": 7, "Sz": 8}
# per-axis factor slots of CutcellKronDesc
F_H, F_K, F_Q, F_S, F_A = range(5)


def _eval(basis: OpenUniformBasis, x: np.ndarray):
    """Dense (n_basis, m) values and derivatives at x (the reference's _eval_all layout)."""
    x = np.asarray(x, dtype=float).ravel()
    e = element_of(basis, x)
    N, D = local_values(basis, e, x)
    V = np.zeros((basis.n_basis, x.size))
    dV = np.zeros((basis.n_basis, x.size))
    cols = np.arange(x.size)
    for i in range(basis.degree + 1):
        V[e + i, cols] = N[:, i]
        dV[e + i, cols] = D[:, i]
    return V, dV


def _panels(basis: OpenUniformBasis, left: float, right: float) -> np.ndarray:
    k = np.unique(basis.knots)
    inner = k[(k > left) & (k < right)]
    return np.unique(np.concatenate(([left], inner, [right])))


def cut_interval_quadrature(basis: OpenUniformBasis, left: float, right: float = 1.0, q: int | None = None):
    """Gauss rule of order max(8, p+4) on every knot panel of [left, right],
    with the basis values and derivatives there (code/cut_3d_sbp.py:351-368)."""
    q = q or max(8, basis.degree + 4)
    g, w = np.polynomial.legendre.leggauss(q)
    pan = _panels(basis, left, right)
    xs, ws = [], []
    for lo, hi in zip(pan[:-1], pan[1:]):
        if hi <= lo:
            continue
        xs.append(0.5 * (hi - lo) * g + 0.5 * (hi + lo))
        ws.append(0.5 * (hi - lo) * w)
    x = np.concatenate(xs)
    wq = np.concatenate(ws)
    V, dV = _eval(basis, x)
    return x, wq, V, dV


@dataclass(frozen=True)
class CutForms1D:
    """1D forms on the cut interval [left, right] (assemble_cut_matrices,
    code/cut_spline_sbp.py:90-146): mass H, advection Q_ij = int phi_i phi_j',
    stiffness K, boundary form S = tR tR^T - tL tL^T, traces and normal
    derivatives at both ends."""

    H: np.ndarray
    Q: np.ndarray
    K: np.ndarray
    S: np.ndarray
    tL: np.ndarray
    tR: np.ndarray
    dL: np.ndarray
    dR: np.ndarray


def cut_interval_forms(basis: OpenUniformBasis, left: float, right: float = 1.0) -> CutForms1D:
    _, w, V, dV = cut_interval_quadrature(basis, left, right)
    H = (V * w) @ V.T
    Q = (V * w) @ dV.T
    K = (dV * w) @ dV.T
    tv, td = _eval(basis, np.array([left, right]))
    tL, tR, dL, dR = tv[:, 0], tv[:, 1], td[:, 0], td[:, 1]
    S = np.outer(tR, tR) - np.outer(tL, tL)
    return CutForms1D(H, Q, K, S, tL, tR, dL, dR)


@dataclass
class AxisFactors:
    """One axis of a cut box: its forms, its 1D extension and the reduced
    factors E^T C E of every form."""

    left: float
    forms: CutForms1D
    E: np.ndarray
    H: np.ndarray
    K: np.ndarray
    Q: np.ndarray
    S: np.ndarray
    F: np.ndarray   # face-trace mass tL tL^T + tR tR^T (reduced)
    N: np.ndarray   # tL (-dL)^T + tR dR^T (reduced): entry (i, j) = phi_i dn phi_j

    @property
    def n(self) -> int:
        return self.E.shape[1]

    def poisson(self, beta: float) -> np.ndarray:
        A = self.K + beta * self.F - self.N - self.N.T
        return 0.5 * (A + A.T)


def axis_factors(basis: OpenUniformBasis, left: float, support_threshold: float = 0.05,
                 preserve_degree: int | None = None) -> AxisFactors:
    f = cut_interval_forms(basis, left)
    E = extension_1d(basis, left, support_threshold, preserve_degree)[0]
    pb = lambda M: E.T @ M @ E
    F = np.outer(f.tL, f.tL) + np.outer(f.tR, f.tR)
    N = np.outer(f.tL, -f.dL) + np.outer(f.tR, f.dR)
    return AxisFactors(left, f, E, pb(f.H), pb(f.K), pb(f.Q), pb(f.S), pb(F), pb(N))


def _kron3(az, ay, ax):
    return np.kron(np.kron(az, ay), ax)


@dataclass
class CutBox:
    """A tensor cut box: basis, per-axis factors (x, y, z) and the weak-penalty
    constant beta = beta_factor (p+1)^2 / h of solve_poisson_3d."""

    basis: OpenUniformBasis
    axes: list
    beta: float

    @property
    def shape(self) -> tuple:
        return tuple(a.n for a in self.axes)

    @property
    def n_red(self) -> int:
        nx, ny, nz = self.shape
        return nx * ny * nz

    def factor(self, axis: int, name: str) -> np.ndarray:
        a = self.axes[axis]
        return a.poisson(self.beta) if name == "A" else getattr(a, name)

    # -- dense forms (CPU, small boxes): the reference's pulled-back matrices
    def dense(self, form: str) -> np.ndarray:
        ax, ay, az = self.axes
        if form == "H":
            return _kron3(az.H, ay.H, ax.H)
        if form in ("K", "A"):
            f = "K" if form == "K" else "A"
            return (_kron3(az.H, ay.H, self.factor(0, f)) + _kron3(az.H, self.factor(1, f), ax.H)
                    + _kron3(self.factor(2, f), ay.H, ax.H))
        d = "xyz".index(form[1])
        kind = form[0]
        parts = [ax.H, ay.H, az.H]
        parts[d] = getattr(self.axes[d], kind)
        return _kron3(parts[2], parts[1], parts[0])

    def diag_A(self) -> np.ndarray:
        ax, ay, az = self.axes
        d = lambda M: np.diag(M).copy()
        return (np.kron(np.kron(d(az.H), d(ay.H)), d(self.factor(0, "A")))
                + np.kron(np.kron(d(az.H), d(self.factor(1, "A"))), d(ax.H))
                + np.kron(np.kron(d(self.factor(2, "A")), d(ay.H)), d(ax.H)))


def cut_box(n_elements: int, degree: int, cut_fractions=(0.6, 0.6, 0.6), beta_factor: float = 12.0,
            support_threshold: float = 0.05, preserve_degree: int | None = None) -> CutBox:
    basis = make_basis(n_elements, degree)
    h = basis.h
    axes = [axis_factors(basis, h * float(f), support_threshold, degree if preserve_degree is None else preserve_degree)
            for f in cut_fractions]
    return CutBox(basis, axes, beta_factor * (degree + 1) ** 2 / h)


# ---------------------------------------------------------------------------
# 3D cut-box Poisson (code/cut_3d_sbp.py:371-531)
# ---------------------------------------------------------------------------


def manufactured_3d():
    """u = exp(0.6 x) cos(pi y) sin(pi z), f = -Lap u (code/cut_3d_sbp.py:371-384)."""

    def u(x, y, z):
        return np.exp(0.6 * x) * np.cos(pi * y) * np.sin(pi * z)

    def f(x, y, z):
        return -(0.36 - 2.0 * pi * pi) * u(x, y, z)

    def grad(x, y, z):
        e = np.exp(0.6 * x)
        return (0.6 * e * np.cos(pi * y) * np.sin(pi * z), -pi * e * np.sin(pi * y) * np.sin(pi * z),
                pi * e * np.cos(pi * y) * np.cos(pi * z))

    return u, f, grad


# Every multi-operand contraction here runs with optimize=True: NumPy then
# contracts one axis at a time through BLAS; without it a four-operand einsum
# is a single loop over all six indices (~1e11 operations at n = 24).


def poisson_rhs(box: CutBox) -> np.ndarray:
    """Reduced load: volume term int f phi plus the face terms
    int_F g (beta phi - dn phi), g = u, on all six faces, pulled back by E."""
    u, _, _ = manufactured_3d()
    quads = [cut_interval_quadrature(box.basis, a.left) for a in box.axes]
    (x, wx, Vx, _), (y, wy, Vy, _), (z, wz, Vz, _) = quads
    # f = -(0.36 - 2 pi^2) exp(0.6 x) cos(pi y) sin(pi z) is a product of 1D
    # factors, so its tensor-quadrature moments are an outer product of three
    # 1D moments (no n_q^3 grid: 512^3 points at n = 64)
    mx = Vx @ (wx * np.exp(0.6 * x))
    my = Vy @ (wy * np.cos(pi * y))
    mz = Vz @ (wz * np.sin(pi * z))
    b = -(0.36 - 2.0 * pi * pi) * mx[:, None, None] * my[None, :, None] * mz[None, None, :]  # (x, y, z)
    lefts = [a.left for a in box.axes]
    for d in range(3):
        o = [j for j in range(3) if j != d]
        a = box.axes[d].forms
        for trace, dtrace, sign, coord in ((a.tL, a.dL, -1.0, lefts[d]), (a.tR, a.dR, 1.0, 1.0)):
            cg = [quads[0][0], quads[1][0], quads[2][0]]
            cg[d] = np.array([coord])
            G = np.squeeze(u(cg[0][:, None, None], cg[1][None, :, None], cg[2][None, None, :]), axis=d)
            fc = np.einsum("ip,jq,pq->ij", quads[o[0]][2] * quads[o[0]][1], quads[o[1]][2] * quads[o[1]][1], G, optimize=True)
            v = box.beta * trace - sign * dtrace
            if d == 0:
                b += np.einsum("a,bc->abc", v, fc)
            elif d == 1:
                b += np.einsum("b,ac->abc", v, fc)
            else:
                b += np.einsum("c,ab->abc", v, fc)
    ax, ay, az = box.axes
    full = np.transpose(b, (2, 1, 0))  # (z, y, x): x fastest
    return np.einsum("zk,yj,xi,zyx->kji", az.E, ay.E, ax.E, full, optimize=True).reshape(-1)


def poisson_errors(box: CutBox, coeff_red: np.ndarray) -> dict:
    """Relative L2 / H1 / L-infinity errors against the manufactured solution on
    the cut-box tensor quadrature (code/cut_3d_sbp.py:506-531)."""
    u, _, grad = manufactured_3d()
    ax, ay, az = box.axes
    nx, ny, nz = box.shape
    c = coeff_red.reshape(nz, ny, nx)
    alpha = np.einsum("zk,yj,xi,kji->zyx", az.E, ay.E, ax.E, c, optimize=True)
    (x, wx, Vx, dVx), (y, wy, Vy, dVy), (z, wz, Vz, dVz) = [cut_interval_quadrature(box.basis, a.left) for a in box.axes]
    # y and z contracted once; the x contraction and the error sums run over
    # slabs of x quadrature points so the n_q^3 grid is never held whole
    t_vv = np.einsum("zyx,yq,zr->xqr", alpha, Vy, Vz, optimize=True)
    t_dv = np.einsum("zyx,yq,zr->xqr", alpha, dVy, Vz, optimize=True)
    t_vd = np.einsum("zyx,yq,zr->xqr", alpha, Vy, dVz, optimize=True)
    nqx = x.size
    sums = np.zeros(4)  # sum W (uh - u)^2, W u^2, W |grad uh - grad u|^2, W |grad u|^2
    linf_num = linf_den = 0.0
    slab = 32
    for p0 in range(0, nqx, slab):
        sl = slice(p0, min(p0 + slab, nqx))
        uh = np.tensordot(Vx[:, sl], t_vv, axes=(0, 0))
        gx = np.tensordot(dVx[:, sl], t_vv, axes=(0, 0))
        gy = np.tensordot(Vx[:, sl], t_dv, axes=(0, 0))
        gz = np.tensordot(Vx[:, sl], t_vd, axes=(0, 0))
        W = wx[sl, None, None] * wy[None, :, None] * wz[None, None, :]
        X, Y, Z = x[sl, None, None], y[None, :, None], z[None, None, :]
        ue = u(X, Y, Z)
        ex, ey, ez = grad(X, Y, Z)
        sums += [np.sum(W * (uh - ue) ** 2), np.sum(W * ue**2),
                 np.sum(W * ((gx - ex) ** 2 + (gy - ey) ** 2 + (gz - ez) ** 2)), np.sum(W * (ex**2 + ey**2 + ez**2))]
        linf_num = max(linf_num, float(np.max(np.abs(uh - ue))))
        linf_den = max(linf_den, float(np.max(np.abs(ue))))
    l2 = np.sqrt(sums[0]) / np.sqrt(sums[1])
    h1 = np.sqrt(sums[2]) / np.sqrt(sums[3])
    linf = linf_num / linf_den
    return {"relative_l2_error": float(l2), "relative_h1_error": float(h1), "relative_linf_error": float(linf)}


def solve_poisson_3d(n_elements: int = 6, degree: int = 3, cut_fractions=(0.6, 0.6, 0.6), beta_factor: float = 12.0,
                     *, linear_solver=None, tol: float = 1e-12, maxiter: int = 20000) -> dict:
    """The reference's cut-box Poisson solve (code/cut_3d_sbp.py:386-531) with
    an opt-in ``linear_solver``:

    * ``None``: dense ``np.linalg.solve`` on the assembled reduced system, as
      the reference does;
    * ``"b200"``: matrix-free Jacobi-PCG on the device (``KronOperator`` +
      ``solve_spd``) to relative residual ``tol``; no N x N matrix is formed;
    * a callable ``(A, b) -> x``: called with the assembled dense system.

    Returns the reference's keys plus ``solver`` (a SolverReport for the
    device path, else None)."""
    box = cut_box(n_elements, degree, cut_fractions, beta_factor)
    rhs = poisson_rhs(box)
    report = None
    if isinstance(linear_solver, str):
        if linear_solver != "b200":
            raise ValueError(f"unknown linear_solver {linear_solver!r}")
        from .fast_solver_backends import solve_spd

        op = KronOperator(box)
        try:
            coeff, report = solve_spd(op, rhs, tol=tol, maxiter=maxiter)
        finally:
            op.close()
    else:
        A = box.dense("A")
        A = 0.5 * (A + A.T)
        coeff = np.linalg.solve(A, rhs) if linear_solver is None else np.asarray(linear_solver(A, rhs))
    out = {"n_elements": n_elements, "degree": degree, "h": box.basis.h, "n_phys": box.n_red}
    out.update(poisson_errors(box, coeff))
    out["solver"] = report
    out["coefficients"] = coeff
    return out


# ---------------------------------------------------------------------------
# device operator
# ---------------------------------------------------------------------------


class CutcellKronDesc(C.Structure):
    _fields_ = [
        ("n", C.c_int32 * 3),
        ("factors", C.c_void_p * 15),  # [axis][H, K, Q, S, A]
        ("diag", C.c_void_p),
    ]


class KronOperator:
    """Matrix-free Kronecker forms of a cut box on the device (libcutcell_b200
    context of kind KRON).  ``solve_device`` solves with the SPD Poisson form
    A; ``apply(x, form)`` applies any of A, H, K, Qx, Qy, Qz, Sx, Sy, Sz."""

    method = "b200-matrix-free-kron-pcg"

    def __init__(self, box: CutBox, device="cuda"):
        import torch

        self.box = box
        self.device = torch.device(device)
        self.n = box.n_red
        self._lib = _lib.load()
        with torch.cuda.device(self.device):
            self._keep = []
            desc = CutcellKronDesc()
            for a in range(3):
                desc.n[a] = box.axes[a].n
                for k, name in enumerate(("H", "K", "Q", "S", "A")):
                    t = torch.as_tensor(np.ascontiguousarray(box.factor(a, name)), dtype=torch.float64,
                                        device=self.device)
                    self._keep.append(t)
                    desc.factors[a * 5 + k] = t.data_ptr()
            d = torch.as_tensor(box.diag_A(), dtype=torch.float64, device=self.device)
            self._keep.append(d)
            desc.diag = d.data_ptr()
            ctx = C.c_void_p()
            _lib.check(self._lib.cutcell_kron_create(C.byref(desc), C.byref(ctx)), "cutcell_kron_create")
            self._ctx = ctx

    def apply(self, x, form: str = "A"):
        import torch

        x = torch.as_tensor(x, dtype=torch.float64, device=self.device).contiguous()
        y = torch.empty_like(x)
        _lib.check(self._lib.cutcell_apply_form(self._ctx, x.data_ptr(), y.data_ptr(), FORMS[form],
                                                _lib.current_stream_ptr()), "cutcell_apply_form")
        return y

    def solve_device(self, b, x=None, *, tol=1e-8, maxiter=5000, precision="fp64", preconditioner="jacobi"):
        import torch

        if precision != "fp64":
            raise ValueError("the Kronecker cut-box operator is solved in FP64")
        b = torch.as_tensor(b, dtype=torch.float64, device=self.device).contiguous()
        if x is None:
            x = torch.empty_like(b)
        rep = _lib.CutcellReport()
        pc = {"none": _lib.PRECOND_NONE, "jacobi": _lib.PRECOND_JACOBI}[preconditioner]
        _lib.check(self._lib.cutcell_pcg_solve(self._ctx, b.data_ptr(), x.data_ptr(), float(tol), int(maxiter),
                                               _lib.FP64, pc, C.byref(rep), _lib.current_stream_ptr()),
                   "cutcell_pcg_solve")
        return x, rep

    def close(self) -> None:
        if getattr(self, "_ctx", None) and self._ctx.value:
            self._lib.cutcell_destroy(self._ctx)
            self._ctx = C.c_void_p()
            self._keep = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
