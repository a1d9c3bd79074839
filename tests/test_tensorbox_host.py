"""Tensor cut box on the host against the reference (tests/golden/tensor_forms.npz,
made by tests/golden/make_golden_tensorbox.py from code/cut_3d_sbp.py and
code/cut_pde_solve.py):

* the pulled-back Kronecker forms H, K, Qx, Qy, Qz, Sx, Sy, Sz, built here
  from per-axis reduced factors, equal the reference's assemble_cut_3d forms
  (compared as products with seeded vectors) to 1e-12 relative;
* the directional Green / SBP residuals ||Q_d + Q_d^T - S_d||_inf are at
  round-off, as the reference's green_residuals_3d;
* solve_poisson_3d with its default dense solve reproduces the reference's
  reduced right-hand side, solution and L2 / H1 / L-infinity errors."""

import numpy as np
import pytest

from cutcell_b200 import tensorbox as tb


@pytest.fixture(scope="module")
def fx(golden):
    return np.load(golden / "tensor_forms.npz")


def test_kronecker_forms_match_reference(fx):
    for k in range(int(fx["n_boxes"])):
        m = fx[f"b{k}_meta"]
        box = tb.cut_box(int(m[0]), int(m[1]), tuple(m[2:]))
        V = fx[f"b{k}_V"]
        assert box.n_red == V.shape[0]
        for name in ("H", "K", "Qx", "Qy", "Qz", "Sx", "Sy", "Sz"):
            ref = fx[f"b{k}_{name}V"]
            got = box.dense(name) @ V
            assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), (k, name)


def test_green_residuals_at_roundoff(fx):
    for k in range(int(fx["n_boxes"])):
        m = fx[f"b{k}_meta"]
        box = tb.cut_box(int(m[0]), int(m[1]), tuple(m[2:]))
        for d, q in enumerate(("Qx", "Qy", "Qz")):
            Q = box.dense(q)
            S = box.dense("S" + q[1])
            r = np.linalg.norm(Q + Q.T - S, ord=np.inf)
            assert r < 1e-14, (k, q, r)
            assert r <= 10 * max(fx[f"b{k}_green"][d], 1e-16)


def test_poisson_3d_matches_reference(fx):
    for k in range(int(fx["n_poisson"])):
        m = fx[f"p{k}_meta"]
        n, p, fr = int(m[0]), int(m[1]), tuple(m[2:])
        box = tb.cut_box(n, p, fr)
        rhs = tb.poisson_rhs(box)
        assert np.linalg.norm(rhs - fx[f"p{k}_rhs"]) <= 1e-12 * np.linalg.norm(fx[f"p{k}_rhs"])
        r = tb.solve_poisson_3d(n, p, fr)
        assert np.linalg.norm(r["coefficients"] - fx[f"p{k}_x"]) <= 1e-9 * np.linalg.norm(fx[f"p{k}_x"])
        np.testing.assert_allclose([r["relative_l2_error"], r["relative_h1_error"], r["relative_linf_error"]],
                                   fx[f"p{k}_err"], rtol=1e-8)
        # a callable linear_solver receives the assembled system
        seen = {}

        def spy(A, b):
            seen["shape"] = A.shape
            return np.linalg.solve(A, b)

        r2 = tb.solve_poisson_3d(n, p, fr, linear_solver=spy)
        assert seen["shape"] == (box.n_red, box.n_red)
        assert np.allclose(r2["coefficients"], r["coefficients"], rtol=0, atol=1e-12 * np.abs(r["coefficients"]).max())
