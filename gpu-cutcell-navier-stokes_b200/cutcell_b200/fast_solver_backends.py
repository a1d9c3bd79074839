"""Drop-in solver backend with the interface of code/fast_solver_backends.py.

``solve_spd(A, b, *, backend, tol, maxiter, preconditioner)`` keeps the
reference signature (code/fast_solver_backends.py:292-300) and its
``SolverReport`` (:30-45); plain FP64 Jacobi-PCG is the default.  The
backend is the hand-written sm_100a library: ``"b200"`` (and the reference's
GPU names ``"gpu"`` / ``"auto"``) run the persistent device PCG.  There is no
CPU solver in this package and no silent fallback: if the library or the GPU
is unavailable the call raises, and solver failures come back as
``success=False`` with the reference's messages.

Extra keywords (defaults keep the reference behaviour):
``precision in {"fp64", "fp32-ir", "bf16-ir"}`` and, for the matrix-free
operator, ``A`` may be a ``CutCellOperator`` (the structured entry).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import asdict, dataclass
from time import perf_counter
from typing import Any, Literal

import numpy as np
import scipy.sparse as sp

from . import _lib

Backend = Literal["b200", "gpu", "auto"]
Preconditioner = Literal["none", "jacobi", "jacobi+learned", "block", "twolevel"]
Precision = Literal["fp64", "fp32-ir", "bf16-ir"]


@dataclass(frozen=True)
class SolverReport:
    """Summary returned by every solver backend (fields of the reference
    report first, device extras after)."""

    backend: str
    method: str
    preconditioner: str
    success: bool
    iterations: int
    elapsed_s: float
    relative_residual: float
    message: str = ""
    transfer_s: float = 0.0
    precision: str = "fp64"
    outer_iterations: int = 1
    device_ms: float = 0.0
    recursive_residual: float = float("nan")

    def to_dict(self) -> dict[str, Any]:
        return asdict(self)


def as_csr(A) -> sp.csr_matrix:
    """``A`` as CSR without changing its values (code/fast_solver_backends.py:48-53)."""
    if sp.issparse(A):
        return A.tocsr()
    return sp.csr_matrix(np.asarray(A, dtype=float))


def csr_memory_bytes(A) -> int:
    Acsr = as_csr(A)
    return int(Acsr.data.nbytes + Acsr.indices.nbytes + Acsr.indptr.nbytes)


class CsrDeviceMatrix:
    """An SPD CSR matrix resident on the device with its solver context."""

    def __init__(self, A, device="cuda"):
        import torch

        Acsr = as_csr(A)
        if Acsr.shape[0] != Acsr.shape[1]:
            raise ValueError("A must be square")
        self.shape = Acsr.shape
        self.n = Acsr.shape[0]
        self.nnz = int(Acsr.nnz)
        self.device = torch.device(device)
        self.indptr = torch.as_tensor(Acsr.indptr.astype(np.int32)).to(self.device)
        self.indices = torch.as_tensor(Acsr.indices.astype(np.int32) if self.nnz else np.zeros(1, np.int32)).to(self.device)
        self.data = torch.as_tensor(Acsr.data.astype(np.float64) if self.nnz else np.zeros(1)).to(self.device)
        self._lib = _lib.load()
        ctx = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(
                self._lib.cutcell_pcg_create_csr(
                    int(self.n), int(self.nnz), self.indptr.data_ptr(), self.indices.data_ptr(), self.data.data_ptr(), C.byref(ctx)
                ),
                "cutcell_pcg_create_csr",
            )
        self._ctx = ctx

    def set_refinement(self, replace_factor: float = 0.1, max_replacements: int = 200) -> None:
        """Controls of the FP32 / BF16 forms (PCG with the reduced-precision
        operator and FP64 residual replacement): the recursive residual is
        replaced by the FP64 true residual each time its norm falls by
        ``replace_factor``; at most ``max_replacements`` replacements."""
        _lib.check(self._lib.cutcell_set_refinement(self._ctx, float(replace_factor), 0, int(max_replacements)), "refinement")

    def apply(self, x, precision: str = "fp64"):
        import torch

        x = torch.as_tensor(x, dtype=torch.float64, device=self.device).contiguous()
        y = torch.empty_like(x)
        _lib.check(
            self._lib.cutcell_apply(self._ctx, x.data_ptr(), y.data_ptr(), _lib.PRECISIONS[precision], _lib.current_stream_ptr()),
            "cutcell_apply",
        )
        return y

    def solve_device(self, b, x=None, *, tol=1e-8, maxiter=5000, precision="fp64", preconditioner="jacobi"):
        import torch

        b = torch.as_tensor(b, dtype=torch.float64, device=self.device).contiguous()
        if x is None:
            x = torch.empty_like(b)
        rep = _lib.CutcellReport()
        pc = {"none": _lib.PRECOND_NONE, "jacobi": _lib.PRECOND_JACOBI}[preconditioner]
        _lib.check(
            self._lib.cutcell_pcg_solve(
                self._ctx, b.data_ptr(), x.data_ptr(), float(tol), int(maxiter), _lib.PRECISIONS[precision], pc,
                C.byref(rep), _lib.current_stream_ptr(),
            ),
            "cutcell_pcg_solve",
        )
        return x, rep

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.cutcell_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _report_from(rep, *, backend, method, preconditioner, precision, tol, elapsed, transfer) -> SolverReport:
    st = int(rep.status)
    rel = float(rep.true_relative_residual)
    success = bool(st == _lib.OK and np.isfinite(rel) and rel <= max(10.0 * tol, 1.0e-14))
    return SolverReport(
        backend=backend,
        method=method,
        preconditioner=preconditioner,
        success=success,
        iterations=int(rep.iterations),
        elapsed_s=float(elapsed),
        relative_residual=rel,
        message=_lib.status_message(st),
        transfer_s=float(transfer),
        precision=precision,
        outer_iterations=int(rep.outer_iterations),
        device_ms=float(rep.elapsed_ms),
        recursive_residual=float(rep.relative_residual),
    )


def solve_b200_cg(
    A,
    b: np.ndarray,
    *,
    tol: float = 1.0e-8,
    maxiter: int = 5000,
    preconditioner: Preconditioner = "jacobi",
    precision: Precision = "fp64",
    replace_factor: float = 0.1,
    device="cuda",
) -> tuple[np.ndarray | None, SolverReport]:
    """Jacobi-PCG on the B200, host arrays in and out (the solve_gpu_cg contract)."""
    import torch

    from .operator import CutCellOperator

    if preconditioner not in ("none", "jacobi"):
        raise ValueError(f"preconditioner {preconditioner!r} needs the learned-preconditioner entry point")
    b_np = np.asarray(b, dtype=float)
    t0 = perf_counter()
    own = False
    if isinstance(A, (CutCellOperator, CsrDeviceMatrix)) or (hasattr(A, "solve_device") and hasattr(A, "n")):
        # device-resident operators (matrix-free tiles, CSR, Kronecker cut boxes)
        dev_op = A
        method = getattr(A, "method", None) or ("b200-matrix-free-pcg" if isinstance(A, CutCellOperator)
                                                else "b200-csr-pcg")
    else:
        dev_op = CsrDeviceMatrix(A, device=device)
        own = True
        method = "b200-csr-pcg"
    if b_np.shape != (dev_op.n,):
        raise ValueError(f"b has shape {b_np.shape}, expected ({dev_op.n},)")
    b_dev = torch.as_tensor(b_np).to(dev_op.device)
    torch.cuda.synchronize(dev_op.device)
    transfer = perf_counter() - t0
    if precision != "fp64":
        dev_op.set_refinement(replace_factor)
    tic = perf_counter()
    x_dev, rep = dev_op.solve_device(b_dev, tol=tol, maxiter=maxiter, precision=precision, preconditioner=preconditioner)
    x = x_dev.cpu().numpy()
    elapsed = perf_counter() - tic
    if own:
        dev_op.close()
    return x, _report_from(
        rep, backend="b200", method=method, preconditioner=preconditioner, precision=precision, tol=tol,
        elapsed=elapsed, transfer=transfer,
    )


def solve_spd(
    A,
    b: np.ndarray,
    *,
    backend: Backend = "b200",
    tol: float = 1.0e-8,
    maxiter: int = 5000,
    preconditioner: Preconditioner = "jacobi",
    precision: Precision = "fp64",
    **kw,
) -> tuple[np.ndarray | None, SolverReport]:
    """Dispatch to the device solver (code/fast_solver_backends.py:292-325)."""
    if backend not in ("b200", "gpu", "auto"):
        raise ValueError(
            f"backend {backend!r} is not provided here: this package only ships the B200 solver "
            "(use the reference's SciPy path for backend='cpu')"
        )
    if preconditioner in ("jacobi+learned", "block", "twolevel"):
        from .learned import solve_learned

        return solve_learned(A, b, tol=tol, maxiter=maxiter, precision=precision, preconditioner=preconditioner, **kw)
    return solve_b200_cg(A, b, tol=tol, maxiter=maxiter, preconditioner=preconditioner, precision=precision, **kw)


def make_linear_solver(*, backend: Backend = "b200", tol: float = 1.0e-13, maxiter: int = 20000,
                       preconditioner: Preconditioner = "jacobi", precision: Precision = "fp64"):
    """A ``linear_solver(A, b) -> x`` callable that routes a wrapper's dense
    ``np.linalg.solve(A, b)`` through ``solve_spd`` (the opt-in
    ``linear_solver=`` of code/cut_3d_sbp.py:503 and
    code/cut_pde_solve.py:446).  A may be dense or sparse and must be SPD; the
    call raises ``RuntimeError`` with the solver's message when the solve does
    not succeed, since those wrappers have no failure path of their own."""

    def linear_solver(A, b):
        x, rep = solve_spd(A, np.asarray(b, dtype=float), backend=backend, tol=tol, maxiter=maxiter,
                           preconditioner=preconditioner, precision=precision)
        if x is None or not rep.success:
            raise RuntimeError(f"linear_solver: {rep.message} (relative residual {rep.relative_residual:.2e})")
        return x

    return linear_solver
