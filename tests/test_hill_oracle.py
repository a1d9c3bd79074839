"""Hill fast-diagonalisation oracle against the reference's own C++ output."""

import numpy as np

from oracle import hill


def test_hill_oracle_matches_reference_fastdiag(golden):
    g = np.load(golden / "hill_fastdiag.npz")
    mu, sig, kap = hill.symbols(g["Mz_row"], g["Sz_row"], g["Kz_row"])
    np.testing.assert_allclose(mu, g["mu"], rtol=0, atol=1e-14 * np.abs(g["mu"]).max())
    np.testing.assert_allclose(sig, g["sig"], rtol=0, atol=1e-12 * np.abs(g["sig"]).max())
    np.testing.assert_allclose(kap, g["kap"], rtol=0, atol=1e-12 * max(1.0, np.abs(g["kap"]).max()))
    Ainv, Sinv = hill.build(g["M2"], g["Qx2"], g["Qy2"], g["KN2"], g["mu"], g["sig"], g["kap"], float(g["a"]))
    out = hill.solve(g["M2"], g["Qx2"], g["Qy2"], g["mu"], g["kap"], Ainv, Sinv, g["ux"], g["uy"], g["uz"])
    for o, ref in zip(out, (g["ox"], g["oy"], g["oz"])):
        assert np.abs(o - ref).max() <= 1e-9 * np.abs(ref).max()


def test_hill_solution_is_weakly_divergence_free(golden):
    """The projected velocity satisfies the weak divergence at round-off
    (the reference's check hill_weak_div, cpp/include/cut/hill3d.h:330-334)."""
    g = np.load(golden / "hill_fastdiag.npz")
    Ainv, Sinv = hill.build(g["M2"], g["Qx2"], g["Qy2"], g["KN2"], g["mu"], g["sig"], g["kap"], float(g["a"]))
    ox, oy, oz = hill.solve(g["M2"], g["Qx2"], g["Qy2"], g["mu"], g["kap"], Ainv, Sinv, g["ux"], g["uy"], g["uz"])
    nz = ox.shape[1]
    Mz = np.array([np.roll(g["Mz_row"], i) for i in range(nz)])
    Kz = np.array([np.roll(g["Kz_row"], i) for i in range(nz)])
    # div = Qx2 ox Mz^T + Qy2 oy Mz^T + M2 oz Kz^T
    div = g["Qx2"] @ ox @ Mz.T + g["Qy2"] @ oy @ Mz.T + g["M2"] @ oz @ Kz.T
    scale = np.abs(g["Qx2"] @ ox @ Mz.T).max()
    assert np.abs(div).max() <= 1e-13  # reference run: 7.9e-15 at ne=6, nz=12
    assert np.abs(div).max() <= 1e-11 * scale
