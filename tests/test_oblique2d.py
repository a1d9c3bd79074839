"""2D oblique-cut host setup against the reference's own outputs (CPU).

Fixtures: tests/golden/oblique2d.npz and oblique_sweep.npz, written by
tests/golden/make_golden_oblique.py from code/oblique_cut_sbp.py and the
committed sweep summary code/results/s6_oblique_sweep_summary.json.
"""

from __future__ import annotations

from math import pi

import numpy as np
import pytest
import scipy.sparse as sp

from cutcell_b200 import oblique2d as ob
from oracle.pcg import cg_loop


@pytest.fixture(scope="module")
def gold(golden):
    return np.load(golden / "oblique2d.npz")


def _case(z, k):
    n, p, ang, frac = z[f"c{k}_meta"][:4]
    n, p = int(n), int(p)
    nrm = np.array([np.cos(ang * pi / 180.0), np.sin(ang * pi / 180.0)])
    nrm /= np.linalg.norm(nrm)
    return n, p, nrm, frac / n


@pytest.mark.parametrize("k", range(4))
def test_forms_match_reference(gold, k):
    n, p, nrm, off = _case(gold, k)
    f = ob.assemble_forms(n, p, nrm, off)
    for name in ("H", "K", "Qx", "Sx"):
        ref = gold[f"c{k}_{name}"]
        got = getattr(f, name)
        scale = np.abs(ref).max()
        assert np.abs(got - ref).max() <= 1e-12 * scale, name
    np.testing.assert_allclose(f.gamma, gold[f"c{k}_gamma"], rtol=1e-12, atol=1e-15)
    # Green identity Qx + Qx^T = Sx (code/oblique_cut_sbp.py:710-713): at the
    # reference's default order it holds to the rule's accuracy, which the
    # reference's own forms show (not exact for p = 5 products)
    ref_res = np.abs(gold[f"c{k}_Qx"] + gold[f"c{k}_Qx"].T - gold[f"c{k}_Sx"]).max()
    assert np.abs(f.Qx + f.Qx.T - f.Sx).max() <= 1e-13 + 2.0 * ref_res
    assert np.abs(f.Qy + f.Qy.T - f.Sy).max() <= 1e-13 + 2.0 * ref_res
    if p < 5:
        assert np.abs(f.Qx + f.Qx.T - f.Sx).max() < 1e-13


@pytest.mark.parametrize("k", range(4))
def test_extension_matches_reference(gold, k):
    n, p, nrm, off = _case(gold, k)
    f = ob.assemble_forms(n, p, nrm, off)
    e = ob.build_extension_2d(f, degree=p)
    np.testing.assert_array_equal(e.interior, gold[f"c{k}_interior"])  # index sets bit-exact
    np.testing.assert_array_equal(e.small_support, gold[f"c{k}_small"])
    Eref = gold[f"c{k}_E"]
    assert e.E.shape == Eref.shape
    np.testing.assert_array_equal(e.E != 0, Eref != 0)
    assert np.abs(e.E - Eref).max() < 1e-9
    assert e.degree == int(gold[f"c{k}_meta"][4])
    assert e.polynomial_residual < 1e-10


@pytest.mark.parametrize("k", range(4))
@pytest.mark.parametrize("form", ["mass", "stiffness"])
def test_reduced_system_and_cg(gold, k, form):
    n, p, nrm, off = _case(gold, k)
    ang = np.arctan2(nrm[1], nrm[0])
    s = ob.build_oblique(n, p, ang, off, form=form)
    pre = f"c{k}_{form}"
    A_ref = sp.csr_matrix((gold[f"{pre}_data"], gold[f"{pre}_indices"], gold[f"{pre}_indptr"]))
    assert s.A.shape == A_ref.shape
    d = abs(s.A - A_ref)
    assert d.max() <= 1e-11 * abs(A_ref).max()
    b = gold[f"{pre}_b"]
    x, rep = cg_loop(s.A, b, tol=1e-9, maxiter=20000)
    it_ref, rel_ref, ok_ref = gold[f"{pre}_rep"]
    assert ok_ref == 1.0 and rep["success"]
    assert abs(rep["iterations"] - it_ref) <= max(1, 0.02 * it_ref)
    xr = gold[f"{pre}_x"]
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-6


def test_sweep_condition_numbers(golden):
    """cond(sym E^T H E) of the reference's 72-row oblique sweep (n = 6,
    p = 3..5, eight angles, three offsets), every sixth row."""
    z = np.load(golden / "oblique_sweep.npz")
    cols = list(z["columns"])
    for row in z["rows"][::6]:
        r = dict(zip(cols, row))
        n, p = int(r["n_elements"]), int(r["p"])
        f = ob.assemble_forms(n, p, [np.cos(r["angle_deg"] * pi / 180), np.sin(r["angle_deg"] * pi / 180)],
                              r["offset_fraction"] / n)
        e = ob.build_extension_2d(f, degree=p)
        Hp = e.E.T @ f.H @ e.E
        Hp = 0.5 * (Hp + Hp.T)
        assert Hp.shape[0] == int(r["n_physical_scalar"])
        ev = np.linalg.eigvalsh(Hp)
        ev = ev[ev > 0]
        assert abs(ev[-1] / ev[0] / r["cond_H_phys"] - 1.0) < 1e-8


def test_sample_cases_draw():
    cases = ob.sample_cases(72, seed=7)
    assert len(cases) == 72
    for n, p, ang, off, form in cases:
        assert n in (6, 8, 12, 16, 24) and p in (3, 4, 5)
        assert 0.0 <= ang <= pi / 4 and 0.0 < off < 1.0 / n
        assert form in ("mass", "stiffness")
    assert ob.sample_cases(72, seed=7) == cases
