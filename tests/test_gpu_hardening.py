"""Input validation and bounded waits of the single-system entry points.

* A malformed CSR (row offsets that fall, a column out of range, wrong end
  offset) is rejected with CUTCELL_E_SHAPE by cutcell_pcg_create_csr before
  any solve reads it.
* Every device-wide wait is bounded: a grid barrier that waits for more
  arrivals than there are blocks gives up after the (runtime) wait limit and
  reports CUTCELL_E_BARRIER, and the device stays usable afterwards.
"""

import ctypes as C
import time

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


def _bad_csrs():
    A = sp.random(50, 50, density=0.1, random_state=3, format="csr") + sp.eye(50, format="csr")
    A = (A + A.T).tocsr()
    ip, ix = A.indptr.astype(np.int32), A.indices.astype(np.int32)
    falling = ip.copy()
    falling[10], falling[11] = falling[11], falling[10] - 1
    col = ix.copy()
    col[7] = 50
    neg = ix.copy()
    neg[3] = -1
    end = ip.copy()
    end[-1] -= 1
    return A, {"falling": (falling, ix), "column": (ip, col), "negative": (ip, neg), "end": (end, ix)}


def test_create_csr_rejects_malformed_structure(torch_cuda):
    from cutcell_b200 import _lib

    torch = torch_cuda
    lib = _lib.load()
    A, cases = _bad_csrs()
    dv = torch.as_tensor(A.data).cuda()
    for name, (ip, ix) in cases.items():
        tip = torch.as_tensor(ip).cuda()
        tix = torch.as_tensor(ix).cuda()
        ctx = C.c_void_p()
        st = lib.cutcell_pcg_create_csr(A.shape[0], A.nnz, tip.data_ptr(), tix.data_ptr(), dv.data_ptr(), C.byref(ctx))
        assert st == _lib.E_SHAPE, name
        assert not ctx.value, name
        assert "malformed" in lib.cutcell_last_error().decode()
    # the well-formed matrix still creates
    tip = torch.as_tensor(A.indptr.astype(np.int32)).cuda()
    tix = torch.as_tensor(A.indices.astype(np.int32)).cuda()
    ctx = C.c_void_p()
    assert lib.cutcell_pcg_create_csr(A.shape[0], A.nnz, tip.data_ptr(), tix.data_ptr(), dv.data_ptr(), C.byref(ctx)) == 0
    assert lib.cutcell_destroy(ctx) == 0


def test_grid_barrier_wait_runs_out_and_reports(torch_cuda):
    from cutcell_b200 import _lib

    lib = _lib.load()
    old = lib.cutcell_get_wait_limit()
    try:
        assert lib.cutcell_set_wait_limit(0.2) == _lib.OK
        status = C.c_int32(-1)
        # a barrier every block reaches completes
        assert lib.cutcell_barrier_selftest(8, 8, C.byref(status)) == _lib.OK
        assert status.value == _lib.OK
        # one arrival more than there are blocks: nothing completes it, the
        # wait gives up after the limit and reports
        t0 = time.perf_counter()
        assert lib.cutcell_barrier_selftest(8, 9, C.byref(status)) == _lib.OK
        dt = time.perf_counter() - t0
        assert status.value == _lib.E_BARRIER
        assert 0.15 < dt < 30.0, dt
        # the device is still usable
        assert lib.cutcell_barrier_selftest(4, 4, C.byref(status)) == _lib.OK
        assert status.value == _lib.OK
    finally:
        lib.cutcell_set_wait_limit(old)
    # a grid that cannot be co-resident is refused, not launched
    assert lib.cutcell_barrier_selftest(1 << 20, 1 << 20, C.byref(status)) == _lib.E_ARG
