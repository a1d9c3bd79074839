"""The allocation-free CSR solve (cutcell_pcg_solve_csr_noalloc) against the
allocating entry point (cutcell_pcg_create_csr + cutcell_pcg_solve), called
through the C ABI.  The allocation-free form exists for callers that cannot
allocate device memory when they solve (a caching allocator holding the
device, loops that must not take cudaMalloc's synchronisation, fixed memory
budgets); its working arrays live in one fixed device array of the library.

This file is collected last so that a run stopping at the first failure has
already run every other test; it must also pass alone in a fresh process."""

import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def _system(golden):
    s = np.load(golden / "stress2d.npz")
    A = sp.csr_matrix((s["s5_data"], s["s5_indices"], s["s5_indptr"]))
    return A, s["s5_b"]


def test_noalloc_solve_matches_allocating_entry_point(torch_cuda, golden):
    from cutcell_b200 import _lib
    from cutcell_b200.fast_solver_backends import CsrDeviceMatrix

    torch = torch_cuda
    lib = _lib.load()
    A, b_np = _system(golden)
    n, nnz = A.shape[0], A.nnz
    ip = torch.as_tensor(A.indptr.astype(np.int32)).cuda()
    ix = torch.as_tensor(A.indices.astype(np.int32)).cuda()
    dv = torch.as_tensor(A.data).cuda()
    b = torch.as_tensor(b_np).cuda()
    tol = 1e-10
    # reference: the allocating context
    dm = CsrDeviceMatrix(A)
    x_ref, rep_ref = dm.solve_device(b, tol=tol, maxiter=5000)
    torch.cuda.synchronize()
    assert rep_ref.status == 0
    # two calls in a row through the allocation-free entry point
    for call in range(2):
        x = torch.full((n,), 123.0, dtype=torch.float64, device="cuda")  # stale contents must not matter
        rep = _lib.CutcellReport()
        st = lib.cutcell_pcg_solve_csr_noalloc(
            n, nnz, ip.data_ptr(), ix.data_ptr(), dv.data_ptr(), b.data_ptr(), x.data_ptr(), tol, 5000,
            _lib.PRECOND_JACOBI, C.byref(rep), _lib.current_stream_ptr(),
        )
        assert st == _lib.OK, lib.cutcell_noalloc_last_error().decode()
        assert rep.status == 0, call
        assert abs(rep.iterations - rep_ref.iterations) <= 1, (call, rep.iterations, rep_ref.iterations)
        assert rep.true_relative_residual <= 10 * tol
        rel = float(torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref))
        assert rel < 1e-9, (call, rel)
    dm.close()


def test_noalloc_rejects_sizes_beyond_its_scratch(torch_cuda):
    from cutcell_b200 import _lib

    lib = _lib.load()
    dummy = torch_cuda.zeros(4, dtype=torch_cuda.float64, device="cuda")
    st = lib.cutcell_pcg_solve_csr_noalloc(
        65537, 65537, dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(),
        1e-8, 10, _lib.PRECOND_JACOBI, None, _lib.current_stream_ptr(),
    )
    assert st == _lib.E_SHAPE
    assert "exceeds" in lib.cutcell_noalloc_last_error().decode()


def _noalloc(lib, _lib, n, nnz, ip, ix, dv, b, x, tol, maxiter, precond, rep):
    return lib.cutcell_pcg_solve_csr_noalloc(
        n, nnz, ip.data_ptr(), ix.data_ptr(), dv.data_ptr(), b.data_ptr(), x.data_ptr(), tol, maxiter, precond,
        C.byref(rep) if rep is not None else None, _lib.current_stream_ptr(),
    )


def test_noalloc_leaves_device_memory_unchanged_and_reports_status(torch_cuda, golden):
    """No device memory is taken by a call (cudaMemGetInfo before and after
    repeated calls, once the first call has resolved the array), solver
    outcomes come back in the report, and the error text is cleared by a
    successful call."""
    from cutcell_b200 import _lib

    torch = torch_cuda
    lib = _lib.load()
    A, b_np = _system(golden)
    n, nnz = A.shape[0], A.nnz
    ip = torch.as_tensor(A.indptr.astype(np.int32)).cuda()
    ix = torch.as_tensor(A.indices.astype(np.int32)).cuda()
    dv = torch.as_tensor(A.data).cuda()
    b = torch.as_tensor(b_np).cuda()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = _lib.CutcellReport()
    assert _noalloc(lib, _lib, n, nnz, ip, ix, dv, b, x, 1e-10, 5000, _lib.PRECOND_JACOBI, rep) == _lib.OK
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    reserved0 = torch.cuda.memory_reserved()
    for _ in range(3):
        assert _noalloc(lib, _lib, n, nnz, ip, ix, dv, b, x, 1e-10, 5000, _lib.PRECOND_JACOBI, rep) == _lib.OK
        assert rep.status == _lib.OK
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    assert torch.cuda.memory_reserved() == reserved0
    assert lib.cutcell_noalloc_last_error().decode() == ""
    # maximum iterations reached: status in the report, the call itself succeeds
    assert _noalloc(lib, _lib, n, nnz, ip, ix, dv, b, x, 1e-14, 3, _lib.PRECOND_JACOBI, rep) == _lib.OK
    assert rep.status == _lib.E_NOCONV and rep.iterations == 3
    # no preconditioner: the same solution as the allocating entry point
    from cutcell_b200.fast_solver_backends import CsrDeviceMatrix

    dm = CsrDeviceMatrix(A)
    x_ref, rep_ref = dm.solve_device(b, tol=1e-10, maxiter=5000, preconditioner="none")
    torch.cuda.synchronize()
    assert _noalloc(lib, _lib, n, nnz, ip, ix, dv, b, x, 1e-10, 5000, _lib.PRECOND_NONE, rep) == _lib.OK
    assert rep.status == _lib.OK and abs(rep.iterations - rep_ref.iterations) <= 1
    assert float(torch.linalg.norm(x - x_ref) / torch.linalg.norm(x_ref)) < 1e-9
    dm.close()


def test_noalloc_rejects_malformed_csr(torch_cuda, golden):
    from cutcell_b200 import _lib

    torch = torch_cuda
    lib = _lib.load()
    A, b_np = _system(golden)
    n, nnz = A.shape[0], A.nnz
    bad_ix = A.indices.astype(np.int32).copy()
    bad_ix[5] = n + 7
    ip = torch.as_tensor(A.indptr.astype(np.int32)).cuda()
    ix = torch.as_tensor(bad_ix).cuda()
    dv = torch.as_tensor(A.data).cuda()
    b = torch.as_tensor(b_np).cuda()
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    rep = _lib.CutcellReport()
    assert _noalloc(lib, _lib, n, nnz, ip, ix, dv, b, x, 1e-10, 100, _lib.PRECOND_JACOBI, rep) == _lib.E_SHAPE
    assert rep.status == _lib.E_SHAPE
    assert "malformed" in lib.cutcell_noalloc_last_error().decode()
    # a bad argument leaves a message too
    assert _noalloc(lib, _lib, n, nnz, ip, ix, dv, b, x, 1e-10, 100, 9, rep) == _lib.E_ARG
    assert "precond" in lib.cutcell_noalloc_last_error().decode()
