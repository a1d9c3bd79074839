"""Device hill advection (hill_skew_conv of all three components) and the
fast step (hill_fastdiag_step) against the oracle and the reference C++.

Tolerances: skew_conv 1e-12 relative to the largest entry (FP64, different
summation order); one full step 1e-9 (it ends in the fast-diagonalisation
solve, whose device/reference agreement is 1e-9 at these sizes)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import hill as ohill

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _adv(m):
    from cutcell_b200.hill import HillAdvection

    return HillAdvection(m["phi"], m["dpx"], m["dpy"], m["w2"], m["Vz"], m["dVz"], m["wz"], m["M2inv"], m["Mzinv"])


def _fd(g):
    from cutcell_b200.hill import FastDiagHill

    return FastDiagHill().build(g["M2"], g["Qx2"], g["Qy2"], g["KN2"], g["Mz_row"], g["Sz_row"], g["Kz_row"], float(g["a"]))


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.fixture(scope="module")
def synth(golden):
    """Synthetic sample machinery on the committed nr = 73, nz = 12 hill
    operators (tests/golden/hill_fastdiag.npz)."""
    from cutcell_b200.hill import synthetic_machinery

    g = np.load(golden / "hill_fastdiag.npz")
    m = synthetic_machinery(nr=int(g["nr"]), nz=int(g["nz"]), cells=(5, 4), pts_per_cell=37, modes_per_row=16,
                            seed=3)
    return g, m


def test_skew_conv_synthetic_vs_oracle(torch_cuda, synth):
    g, m = synth
    adv = _adv(m)
    try:
        u = [g["ux"], g["uy"], g["uz"]]
        out = [o.cpu().numpy() for o in adv.skew_conv(*u)]
        wq = [ohill.sample(m["phi"], c, m["Vz"]) for c in u]
        for o, c in zip(out, u):
            assert _rel(o, ohill.skew_conv(m, wq, c)) < 1e-12
        again = [o.cpu().numpy() for o in adv.skew_conv(*u)]
        for a, b in zip(out, again):
            np.testing.assert_array_equal(a, b)  # fixed-order gather: same bits
    finally:
        adv.close()


def test_step_synthetic_vs_oracle(torch_cuda, synth):
    g, m = synth
    adv, fd = _adv(m), _fd(g)
    try:
        u = [torch_cuda.as_tensor(g[k]).cuda().contiguous() for k in ("ux", "uy", "uz")]
        adv.step(fd, u, 0.02, 0.7)
        got = [t.cpu().numpy() for t in u]
        Ainv, Sinv = ohill.build(g["M2"], g["Qx2"], g["Qy2"], g["KN2"], g["mu"], g["sig"], g["kap"], float(g["a"]))
        fdo = dict(M2=g["M2"], Qx2=g["Qx2"], Qy2=g["Qy2"], mu=g["mu"], kap=g["kap"], Ainv=Ainv, Sinv=Sinv)
        want = ohill.fast_step(m, fdo, [g["ux"], g["uy"], g["uz"]], 0.02, 0.7)
        for a, b in zip(got, want):
            assert _rel(a, b) < 1e-9
    finally:
        adv.close()
        fd.close()


@pytest.fixture(scope="module")
def refm():
    d = ohill.reference_dump(3, 6, seed=99, steps=1)
    if d is None:
        pytest.skip("reference hill binary unavailable (oracle/_ref/hill_ref)")
    return d


def test_skew_conv_reference_machinery(torch_cuda, refm):
    adv = _adv(refm)
    try:
        out = [o.cpu().numpy() for o in adv.skew_conv(refm["ux"], refm["uy"], refm["uz"])]
        for o, name in zip(out, ("cx", "cy", "cz")):
            assert _rel(o, refm[name]) < 1e-12
    finally:
        adv.close()


def test_step_reference_machinery(torch_cuda, refm):
    adv, fd = _adv(refm), _fd(refm)
    try:
        u = [torch_cuda.as_tensor(refm[k]).cuda().contiguous() for k in ("ux", "uy", "uz")]
        adv.step(fd, u, 0.02, 0.7)
        for t, name in zip(u, ("sx", "sy", "sz")):
            assert _rel(t.cpu().numpy(), refm[name]) < 1e-9
    finally:
        adv.close()
        fd.close()


def test_unsupported_shapes_rejected(torch_cuda):
    from cutcell_b200 import _lib
    from cutcell_b200.hill import synthetic_machinery

    m = synthetic_machinery(nr=64, nz=40, cells=(2, 2), pts_per_cell=4, modes_per_row=8)
    with pytest.raises(_lib.CutcellLibraryError):
        _adv(m)
