"""Hill advection / fast-step oracle against the reference C++ (CPU), and the
host tables of the device advection.

The reference machinery (sparse 2D sample rows, z basis, mass inverses) is
produced at test time by oracle/_ref/hill_ref, compiled from the
reference's own headers (oracle/build_ref.py); the tests skip when that
binary cannot be built or found."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import hill


@pytest.fixture(scope="module")
def ref():
    d = hill.reference_dump(3, 6, seed=99, steps=1)
    if d is None:
        pytest.skip("reference hill binary unavailable")
    return d


def test_skew_conv_matches_reference(ref):
    u = [ref["ux"], ref["uy"], ref["uz"]]
    wq = [hill.sample(ref["phi"], c, ref["Vz"]) for c in u]
    for c, name in zip(u, ("cx", "cy", "cz")):
        got = hill.skew_conv(ref, wq, c)
        assert np.abs(got - ref[name]).max() <= 1e-13 * np.abs(ref[name]).max()


def test_fast_step_matches_reference(ref):
    Ainv, Sinv = hill.build(ref["M2"], ref["Qx2"], ref["Qy2"], ref["KN2"], ref["mu"], ref["sig"], ref["kap"], ref["a"])
    fd = dict(M2=ref["M2"], Qx2=ref["Qx2"], Qy2=ref["Qy2"], mu=ref["mu"], kap=ref["kap"], Ainv=Ainv, Sinv=Sinv)
    out = hill.fast_step(ref, fd, [ref["ux"], ref["uy"], ref["uz"]], 0.02, 0.7)
    for o, name in zip(out, ("sx", "sy", "sz")):
        assert np.abs(o - ref[name]).max() <= 1e-10 * np.abs(ref[name]).max()


def test_device_tables_from_reference_machinery(ref):
    from cutcell_b200.hill import segment_tables, z_element_tables

    nz = ref["nz"]
    zb, Vl, dVl, wzl, qpe = z_element_tables(ref["Vz"], ref["dVz"], ref["wz"], nz)
    assert zb.shape == (nz, 4) and qpe * nz == ref["Vz"].shape[0]
    for j in range(4):  # scatter round j writes distinct modes
        assert len(set(zb[:, j])) == nz
    # the band reproduces Vz exactly
    for e in range(nz):
        full = np.zeros((qpe, nz))
        full[:, zb[e]] = Vl[e]
        np.testing.assert_array_equal(full, ref["Vz"][e * qpe : (e + 1) * qpe])
    P = ref["phi"]
    t = segment_tables(P.indptr, P.indices, seg_max=128)
    q0, q1 = t["seg_q0"], t["seg_q1"]
    assert q0[0] == 0 and q1[-1] == P.shape[0] and np.all(q0[1:] == q1[:-1]) and np.all(q1 - q0 <= 128)
    for s in range(q0.size):
        pat = t["pat_idx"][t["seg_pat"][s] : t["seg_pat"][s] + t["seg_len"][s]]
        for q in (q0[s], q1[s] - 1):
            np.testing.assert_array_equal(P.indices[P.indptr[q] : P.indptr[q + 1]], pat)
    # every partial row is gathered exactly once, into its own mode
    g_ptr, g_ent = t["g_ptr"], t["g_ent"]
    assert np.array_equal(np.sort(g_ent), np.arange(t["pat_idx"].size))
    for m in range(g_ptr.size - 1):
        ent = g_ent[g_ptr[m] : g_ptr[m + 1]]
        assert np.all(t["pat_idx"][ent] == m) and np.all(np.diff(ent) > 0)


def test_synthetic_machinery_shapes():
    from cutcell_b200.hill import synthetic_machinery, z_element_tables

    m = synthetic_machinery(nr=300, nz=8, cells=(4, 3), pts_per_cell=10)
    assert m["phi"].shape == (120, 300) and m["Vz"].shape == (72, 8)
    zb, *_ = z_element_tables(m["Vz"], m["dVz"], m["wz"], 8)
    assert zb.shape == (8, 4)
    # partition of unity of the periodic cubic B-splines
    np.testing.assert_allclose(m["Vz"].sum(1), 1.0, atol=1e-14)
    np.testing.assert_allclose(m["dVz"].sum(1), 0.0, atol=1e-12)
