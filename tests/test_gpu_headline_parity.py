"""Parity at the headline configuration: the sphere-cut Poisson problem,
r = 0.31, p = 3, n = 32 (39,684 reduced unknowns), the workload the bench
times.  The oracle assembles E^T A E independently (oracle/assembly.py,
element by element as code/bell_3d_core.py does) and solves it with its CG
restatement (oracle/pcg.py) to tol 1e-13.

Bars (relative L2 against the oracle's tol-1e-13 solution):
* FP64 matrix-free Jacobi-PCG to tol 1e-13: <= 1e-9, and at tol 1e-9 its
  iteration count is within max(1, 2 %) of the oracle CG's;
* the FP32 and two-plane BF16 operator forms (PCG with FP64 residual
  replacement) to tol 1e-11: <= 1e-7; at tol 1e-9 they converge within 5 %
  of plain FP64's iterations.
The inner iteration counts of every form are printed beside plain's."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def headline():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    from cutcell_b200.workloads import sphere_poisson
    from oracle.aggregation import restrict_spd
    from oracle.assembly import assemble_full
    from oracle.pcg import cg_loop

    prob, ext = sphere_poisson(32, 3, 0.31)
    b = np.asarray(ext.E.T @ prob.load)
    A = restrict_spd(assemble_full(prob), ext.E).tocsr()
    x_ref, rep_ref = cg_loop(A, b, tol=1e-13, maxiter=50000)
    _, rep9 = cg_loop(A, b, tol=1e-9, maxiter=50000)
    return prob, ext, b, x_ref, rep9["iterations"]


def test_headline_fp64_and_mixed_forms_match_oracle(headline):
    from cutcell_b200 import solve_spd
    from cutcell_b200.operator import CutCellOperator

    prob, ext, b, x_ref, it_oracle = headline
    assert ext.n_red == 39684
    op = CutCellOperator(prob, ext)
    err = lambda x: float(np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref))
    try:
        x9, r9 = solve_spd(op, b, tol=1e-9, maxiter=20000)
        assert r9.success, r9
        assert abs(r9.iterations - it_oracle) <= max(1, 0.02 * it_oracle), (r9.iterations, it_oracle)
        x13, r13 = solve_spd(op, b, tol=1e-13, maxiter=20000)
        assert r13.success, r13
        assert err(x13) <= 1e-9, err(x13)
        its = {"oracle": it_oracle, "fp64": r9.iterations}
        for prec in ("fp32-ir", "bf16-ir"):
            _, m9 = solve_spd(op, b, tol=1e-9, maxiter=20000, precision=prec)
            assert m9.success, (prec, m9)
            its[prec] = m9.iterations
            assert m9.iterations <= 1.05 * r9.iterations, (prec, m9.iterations, r9.iterations)
            x11, m11 = solve_spd(op, b, tol=1e-11, maxiter=20000, precision=prec)
            assert m11.success, (prec, m11)
            assert err(x11) <= 1e-7, (prec, err(x11))
        print("headline iterations at tol 1e-9:", its)
    finally:
        op.close()
