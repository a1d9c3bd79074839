"""Parity of the device solve path with the CPU oracle (needs a B200)."""

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from oracle import pcg as op

from _systems import system

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _stress(golden, k):
    s = np.load(golden / "stress2d.npz")
    A = sp.csr_matrix((s[f"s{k}_data"], s[f"s{k}_indices"], s[f"s{k}_indptr"]))
    return A, s[f"s{k}_b"], s[f"s{k}_x"], s[f"s{k}_meta"]


@pytest.mark.parametrize("k", range(7))
def test_csr_pcg_matches_reference_golden(torch_cuda, golden, k):
    from cutcell_b200 import solve_spd

    A, b, xref, meta = _stress(golden, k)
    x, rep = solve_spd(A, b, backend="b200", tol=1e-8, maxiter=5000)
    assert rep.success, rep
    assert abs(rep.iterations - int(meta[3])) <= 1  # iteration counts within one
    assert rep.relative_residual < 1e-8
    assert np.linalg.norm(x - xref) / np.linalg.norm(xref) < 1e-7
    # tighter solve against a direct solve: FP64 parity 1e-9
    x2, rep2 = solve_spd(A, b, backend="b200", tol=1e-13, maxiter=20000)
    xd = spla.spsolve(A.tocsc(), b)
    assert np.linalg.norm(x2 - xd) / np.linalg.norm(xd) < 1e-9


def test_csr_pcg_deterministic(torch_cuda, golden):
    from cutcell_b200.fast_solver_backends import CsrDeviceMatrix

    A, b, _, _ = _stress(golden, 5)
    dm = CsrDeviceMatrix(A)
    bt = torch_cuda.as_tensor(b).cuda()
    x1, r1 = dm.solve_device(bt, tol=1e-10)
    x2, r2 = dm.solve_device(bt, tol=1e-10)
    assert r1.iterations == r2.iterations
    assert torch_cuda.equal(x1, x2)
    dm.close()


def test_csr_edge_cases(torch_cuda):
    from cutcell_b200 import solve_spd

    A = sp.diags([2.0, 3.0, 4.0, 5.0], format="csr")
    b = np.array([1.0, -2.0, 0.5, 4.0])
    x, rep = solve_spd(A, b, tol=1e-12, maxiter=20)
    assert rep.success and rep.relative_residual < 1e-10  # test_fast_solver_backends.py:10-16
    np.testing.assert_allclose(A @ x, b, rtol=1e-10, atol=1e-12)
    # maxiter exhausted
    A2, b2 = sp.diags([1.0, 10.0, 100.0, 1000.0], format="csr"), np.ones(4)
    x, rep = solve_spd(A2, b2, tol=1e-14, maxiter=1, preconditioner="none")
    assert not rep.success and rep.message == "maximum iterations reached" and rep.iterations == 1
    # indefinite -> breakdown, like the reference loop
    x, rep = solve_spd(sp.diags([1.0, -1.0], format="csr"), np.array([0.0, 1.0]), tol=1e-12)
    assert not rep.success and rep.message.startswith("CG breakdown")
    # zero RHS: breakdown at k = 1 with x = 0 (code/fast_solver_backends.py:249-256)
    x, rep = solve_spd(A, np.zeros(4), tol=1e-12)
    assert np.all(x == 0) and rep.iterations == 1
    # NaN RHS
    x, rep = solve_spd(A, np.array([1.0, np.nan, 0.0, 0.0]), tol=1e-12)
    assert not rep.success
    # single unknown
    x, rep = solve_spd(sp.csr_matrix(np.array([[4.0]])), np.array([2.0]), tol=1e-14)
    assert rep.success and abs(x[0] - 0.5) < 1e-15


CASES = [("sphere", 6, 2), ("plane", 6, 3), ("sphere", 9, 3), ("sphere", 8, 4), ("plane", 5, 5)]


@pytest.mark.parametrize("kind,n,p", CASES)
def test_matrix_free_apply_matches_oracle(torch_cuda, kind, n, p):
    from cutcell_b200.operator import CutCellOperator

    prob, ext, A_full, A_red, b = system(kind, n, p)
    op_ = CutCellOperator(prob, ext)
    rng = np.random.default_rng(7)
    x = rng.standard_normal(ext.n_red)
    ref = A_red @ x
    for prec, tol in (("fp64", 1e-12), ("fp32-ir", 1e-5), ("bf16-ir", 2e-2)):
        y = op_.apply(x, prec).cpu().numpy()
        assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < tol, prec
    # E gather / scatter
    xf = op_.gather(x).cpu().numpy()
    np.testing.assert_allclose(xf, ext.E @ x, rtol=1e-14, atol=1e-14)
    yf = rng.standard_normal(ext.n_full)
    yr = op_.scatter(yf).cpu().numpy()
    np.testing.assert_allclose(yr, ext.E.T @ yf, rtol=1e-13, atol=1e-13)
    # identity rows are copied bit-exactly
    assert np.array_equal(xf[ext.interior], x)
    op_.close()


def test_matrix_free_apply_three_tiles_per_axis(torch_cuda):
    """p = 5: the 9-wide tile windows overlap so that interior DOFs lie in
    three tiles per axis (27 partial slots); n = 10 has three tiles per axis."""
    from cutcell_b200.operator import CutCellOperator

    prob, ext, A_full, A_red, b = system("plane", 10, 5)
    op_ = CutCellOperator(prob, ext)
    assert op_.layout.n_tiles_axis == 3
    x = np.random.default_rng(9).standard_normal(ext.n_red)
    ref = A_red @ x
    y = op_.apply(x, "fp64").cpu().numpy()
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-12
    op_.close()


@pytest.mark.parametrize("kind,n,p", CASES[:3])
def test_matrix_free_pcg_matches_oracle(torch_cuda, kind, n, p):
    from cutcell_b200 import solve_spd
    from cutcell_b200.operator import CutCellOperator

    prob, ext, A_full, A_red, b = system(kind, n, p)
    op_ = CutCellOperator(prob, ext)
    _, rep_o = op.cg_loop(A_red, b, tol=1e-9, maxiter=20000)
    x, rep = solve_spd(op_, b, tol=1e-9, maxiter=20000)
    assert rep.success, rep
    # round-off in the summation order only: within one iteration, or 2 % on
    # ill-conditioned systems that need hundreds of iterations
    assert abs(rep.iterations - rep_o["iterations"]) <= max(1, 0.02 * rep_o["iterations"])
    xd = spla.spsolve(A_red.tocsc(), b)
    x2, rep2 = solve_spd(op_, b, tol=1e-13, maxiter=20000)
    assert np.linalg.norm(x2 - xd) / np.linalg.norm(xd) < 1e-9
    if p < 3:
        # reduced-precision refinement is built for p >= 3 only
        from cutcell_b200._lib import CutcellLibraryError

        with pytest.raises(CutcellLibraryError):
            solve_spd(op_, b, tol=1e-9, precision="fp32-ir")
        op_.close()
        return
    # reduced-precision operator with FP64 residual replacement: converges to
    # the same tolerance, with the FP64 solution's accuracy (1e-7 at tol 1e-11)
    # and an iteration count near plain FP64's
    for prec in ("fp32-ir", "bf16-ir"):
        x3, rep3 = solve_spd(op_, b, tol=1e-9, maxiter=20000, precision=prec)
        assert rep3.success, (prec, rep3)
        factor = {"fp32-ir": 1.35, "bf16-ir": 1.7}[prec]  # as in the sliver-stress set
        assert rep3.relative_residual <= 1e-8 and rep3.iterations <= factor * rep.iterations + 5, (prec, rep3, rep)
        x4, rep4 = solve_spd(op_, b, tol=1e-11, maxiter=20000, precision=prec)
        assert rep4.success, (prec, rep4)
        assert np.linalg.norm(x4 - xd) / np.linalg.norm(xd) < 1e-7
    op_.close()
