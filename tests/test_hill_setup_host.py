"""The restated hill build (cutcell_b200.hillsetup.build_hill) against the
reference's own Hill3D::build (cpp/include/cut/hill3d.h:95-171), run through
oracle/_ref/hill_ref (compiled from the reference's headers by
oracle/build_ref.py; these tests skip where it is unavailable):

* at nex = ney the reduced forms M2, Qx2, Qy2, KN2, M2inv, the periodic z
  forms, the sparse sample rows (pattern bit-exact, values 1e-12) and the
  quadrature tables equal the reference's, in the unit-square and in the
  physical metric;
* on an anisotropic grid (nex = 2 ney) the extension reproduces every
  polynomial of total degree <= p on the active functions, M2 and KN2 are
  symmetric positive definite, and one oracle fast step drives the weak
  divergence of the parabolic initial condition to round-off."""

import numpy as np
import pytest

from cutcell_b200.hillsetup import build_hill, parabolic_ic, weak_div


def _dump(ne, nz, physical):
    from oracle import hill as oh

    d = oh.reference_dump(ne, nz, seed=99, steps=0, physical=physical)
    if d is None:
        pytest.skip("reference hill binary unavailable")
    return d


@pytest.mark.parametrize("ne,nz,physical", [(3, 6, False), (5, 8, True)])
def test_build_matches_reference(ne, nz, physical):
    d = _dump(ne, nz, physical)
    hs = build_hill(ne, ne, 3, nz, 4.5, physical=physical)
    rel = lambda a, b: np.abs(a - b).max() / np.abs(b).max()
    assert hs.nr == d["nr"]
    for k in ("M2", "Qx2", "Qy2", "KN2", "M2inv", "Mzinv"):
        assert rel(getattr(hs, k), d[k]) < 1e-12, k
    assert rel(hs.Mz[0], d["Mz_row"]) < 1e-13 and rel(hs.Sz[0], d["Sz_row"]) < 1e-13
    assert rel(hs.Kz[0], d["Kz_row"]) < 1e-13
    for k in ("phi", "dpx", "dpy"):
        A, B = getattr(hs, k), d[k]
        assert np.array_equal(A.indptr, B.indptr) and np.array_equal(A.indices, B.indices), k
        assert np.abs(A.data - B.data).max() <= 1e-12 * np.abs(B.data).max(), k
    for k in ("w2", "Vz", "dVz", "wz"):
        assert rel(getattr(hs, k), d[k]) < 1e-12, k


def test_anisotropic_build_properties():
    from oracle import hill as oh
    from cutcell_b200.hill import mode_inverses, z_symbols

    hs = build_hill(16, 8, 3, 8, 4.5, physical=True)
    B = hs.forms.basis
    poly = B.poly(3)
    active = hs.gamma > 1e-22
    for row in poly:
        assert np.abs(hs.E @ row[hs.interior] - row * active).max() < 1e-9
    for M in (hs.M2, hs.KN2):
        assert np.abs(M - M.T).max() <= 1e-12 * np.abs(M).max()
        assert np.linalg.eigvalsh(0.5 * (M + M.T)).min() > 0
    mu, sig, kap = z_symbols(hs.Mz[0], hs.Sz[0], hs.Kz[0])
    Ai, Si = mode_inverses(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, mu, sig, kap, 0.02 / 5600)
    fd = dict(M2=hs.M2, Qx2=hs.Qx2, Qy2=hs.Qy2, mu=mu, kap=kap, Ainv=Ai, Sinv=Si)
    u0 = parabolic_ic(hs)
    u1 = oh.fast_step(hs.machinery(), fd, list(u0), 0.02, 0.0)
    d0, d1 = np.abs(weak_div(hs, *u0)).max(), np.abs(weak_div(hs, *u1)).max()
    assert d1 <= 1e-10 * d0, (d0, d1)
