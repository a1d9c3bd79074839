"""Device fast-diagonalisation solve against the reference's FastDiagHill
(golden vectors from the reference C++; needs a B200)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def test_fastdiag_solve_matches_reference(torch_cuda, golden):
    from cutcell_b200.hill import FastDiagHill

    g = np.load(golden / "hill_fastdiag.npz")
    fd = FastDiagHill().build(g["M2"], g["Qx2"], g["Qy2"], g["KN2"], g["Mz_row"], g["Sz_row"], g["Kz_row"], float(g["a"]))
    np.testing.assert_allclose(fd.mu, g["mu"], rtol=0, atol=1e-14 * np.abs(g["mu"]).max())
    out = fd.solve(g["ux"], g["uy"], g["uz"])
    for o, ref in zip(out, (g["ox"], g["oy"], g["oz"])):
        assert np.abs(o - ref).max() <= 1e-9 * np.abs(ref).max()
    # weak divergence of the projected velocity at round-off (reference: 7.9e-15)
    nz = out[0].shape[1]
    Mz = np.array([np.roll(g["Mz_row"], i) for i in range(nz)])
    Kz = np.array([np.roll(g["Kz_row"], i) for i in range(nz)])
    div = g["Qx2"] @ out[0] @ Mz.T + g["Qy2"] @ out[1] @ Mz.T + g["M2"] @ out[2] @ Kz.T
    assert np.abs(div).max() <= 1e-13
    # repeated solves are bit-identical (no atomics)
    out2 = fd.solve(g["ux"], g["uy"], g["uz"])
    assert all(np.array_equal(a, b) for a, b in zip(out, out2))
    fd.close()
