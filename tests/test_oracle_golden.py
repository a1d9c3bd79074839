"""The CPU oracle against golden vectors produced by the reference's own code."""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import aggregation as oa
from oracle import pcg as op


def _csr(g, prefix=""):
    return sp.csr_matrix((g[prefix + "data"], g[prefix + "indices"], g[prefix + "indptr"]))


@pytest.mark.parametrize("name", ["ext3d_sphere", "ext3d_bell"])
def test_oracle_extension_bit_exact(golden, name):
    g = np.load(golden / f"{name}.npz")
    Eref = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"]))
    E, interior, small = oa.extension_3d(g["gamma"], int(g["n"]), int(g["p"]))
    assert np.array_equal(interior, g["interior"])
    assert np.array_equal(small, g["small"])
    assert np.array_equal(E.indptr, Eref.indptr) and np.array_equal(E.indices, Eref.indices)
    assert abs(E - Eref).max() <= 1e-12


def test_bell_unknown_count_matches_published(golden):
    # benchmarks/README.md:23 -- 20 elements per axis, 9,832 unknowns
    g = np.load(golden / "ext3d_bell.npz")
    assert int(g["shape"][1]) == 9832


def test_oracle_cg_matches_reference_iterations(golden):
    s = np.load(golden / "stress2d.npz")
    for k in range(int(s["count"])):
        A = sp.csr_matrix((s[f"s{k}_data"], s[f"s{k}_indices"], s[f"s{k}_indptr"]))
        b = s[f"s{k}_b"]
        p, n, eps, it_ref, rel_ref, n_red, nnz = s[f"s{k}_meta"]
        x, rep = op.solve_cpu_cg(A, b, tol=1e-8)
        assert rep["iterations"] == int(it_ref)
        assert rep["success"]
        np.testing.assert_allclose(x, s[f"s{k}_x"], rtol=0, atol=1e-12 * np.abs(s[f"s{k}_x"]).max())
        x2, rep2 = op.cg_loop(A, b, tol=1e-8)
        assert abs(rep2["iterations"] - int(it_ref)) <= 1
        assert rep2["relative_residual"] < 1e-8


def test_stress_shapes_match_reference_csv(golden):
    # code/results/fast_solver_stress.csv: n=8 p=4 -> 120 unknowns, 7,396 nnz
    s = np.load(golden / "stress2d.npz")
    p, n, eps, it_ref, rel_ref, n_red, nnz = s["s0_meta"]
    assert (int(n_red), int(nnz)) == (120, 7396)
    assert int(it_ref) == 105


def test_cg_loop_edge_cases():
    A = sp.diags([2.0, 3.0, 4.0, 5.0], format="csr")
    b = np.array([1.0, -2.0, 0.5, 4.0])
    x, rep = op.cg_loop(A, b, tol=1e-12, maxiter=20)
    assert rep["success"]
    x, rep = op.cg_loop(A, np.zeros(4), tol=1e-12, maxiter=20)
    assert rep["iterations"] == 1 or rep["message"] != "converged" or np.all(x == 0)
    x, rep = op.cg_loop(sp.diags([1.0, -1.0], format="csr"), np.array([0.0, 1.0]), tol=1e-12)
    assert rep["message"].startswith("CG breakdown")
