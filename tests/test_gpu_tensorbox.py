"""Matrix-free Kronecker forms of tensor cut boxes on the device, and the
two Poisson wrappers routed through solve_spd (tests/golden/tensor_forms.npz,
made from code/cut_3d_sbp.py and code/cut_pde_solve.py):

* cutcell_apply_form reproduces the reference's pulled-back H, K, Qx, Qy, Qz,
  Sx, Sy, Sz (products with seeded vectors) to 1e-12 relative;
* the directional Green identity holds on the device to round-off:
  <v, Q_d u> + <u, Q_d v> = <v, S_d u> (code/cut_3d_sbp.py:149-154);
* solve_poisson_3d(linear_solver="b200") solves matrix-free to tol 1e-13 and
  matches the reference's dense-solve coefficients to 1e-9 and its errors to
  1e-7 relative;
* solve_poisson_circular's captured system, solved through
  make_linear_solver(), matches the reference's np.linalg.solve to 1e-9;
* at n = 24 the Kronecker Poisson operator matches a host sum-factorised
  evaluation to 1e-12 and its Jacobi-PCG agrees with the same iteration on
  the host."""

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


@pytest.fixture(scope="module")
def fx(golden):
    return np.load(golden / "tensor_forms.npz")


def _host_apply(box, form, x):
    """Sum-factorised host evaluation of a form (x fastest)."""
    nx, ny, nz = box.shape
    X = x.reshape(nz, ny, nx)
    ax, ay, az = box.axes

    def prod(cz, cy, cx):  # three passes, one axis at a time
        t = np.einsum("ck,ijk->ijc", cx, X)
        t = np.einsum("bj,ijc->ibc", cy, t)
        return np.einsum("ai,ibc->abc", cz, t)

    if form in ("A", "K"):
        f = [box.factor(d, form) for d in range(3)]
        y = prod(az.H, ay.H, f[0]) + prod(az.H, f[1], ax.H) + prod(f[2], ay.H, ax.H)
    elif form == "H":
        y = prod(az.H, ay.H, ax.H)
    else:
        d = "xyz".index(form[1])
        parts = [ax.H, ay.H, az.H]
        parts[d] = getattr(box.axes[d], form[0])
        y = prod(parts[2], parts[1], parts[0])
    return y.reshape(-1)


def test_apply_forms_match_reference(torch_cuda, fx):
    from cutcell_b200 import tensorbox as tb

    for k in range(int(fx["n_boxes"])):
        m = fx[f"b{k}_meta"]
        box = tb.cut_box(int(m[0]), int(m[1]), tuple(m[2:]))
        op = tb.KronOperator(box)
        V = fx[f"b{k}_V"]
        for name in ("H", "K", "Qx", "Qy", "Qz", "Sx", "Sy", "Sz"):
            ref = fx[f"b{k}_{name}V"]
            got = np.stack([op.apply(V[:, j], name).cpu().numpy() for j in range(V.shape[1])], axis=1)
            assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), (k, name)
        # Green identity on the device
        u, v = V[:, 0], V[:, 1]
        for d in "xyz":
            Qu, Qv, Su = (op.apply(w, f).cpu().numpy() for w, f in ((u, "Q" + d), (v, "Q" + d), (u, "S" + d)))
            lhs = v @ Qu + u @ Qv
            scale = np.linalg.norm(v) * np.linalg.norm(Qu) + np.linalg.norm(v) * np.linalg.norm(Su)
            assert abs(lhs - v @ Su) <= 1e-13 * scale, (k, d)
        op.close()


def test_poisson_3d_routed_through_solve_spd(torch_cuda, fx):
    from cutcell_b200 import tensorbox as tb

    for k in range(int(fx["n_poisson"])):
        m = fx[f"p{k}_meta"]
        r = tb.solve_poisson_3d(int(m[0]), int(m[1]), tuple(m[2:]), linear_solver="b200", tol=1e-13)
        rep = r["solver"]
        assert rep is not None and rep.success, rep
        x_ref = fx[f"p{k}_x"]
        assert np.linalg.norm(r["coefficients"] - x_ref) <= 1e-9 * np.linalg.norm(x_ref)
        np.testing.assert_allclose([r["relative_l2_error"], r["relative_h1_error"], r["relative_linf_error"]],
                                   fx[f"p{k}_err"], rtol=1e-7)


def test_circular_poisson_system_routed_through_solve_spd(torch_cuda, fx):
    from cutcell_b200 import make_linear_solver

    solve = make_linear_solver(tol=1e-13)
    for k in range(int(fx["n_circular"])):
        A = sp.csr_matrix((fx[f"c{k}_data"], fx[f"c{k}_indices"], fx[f"c{k}_indptr"]))
        x = solve(A, fx[f"c{k}_rhs"])
        x_ref = fx[f"c{k}_x"]
        assert np.linalg.norm(x - x_ref) <= 1e-9 * np.linalg.norm(x_ref), k


def test_kron_poisson_at_scale(torch_cuda):
    import torch

    from cutcell_b200 import solve_spd
    from cutcell_b200 import tensorbox as tb

    box = tb.cut_box(24, 3, (0.7, 0.2, 0.95))
    op = tb.KronOperator(box)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(box.n_red)
    for form in ("A", "H", "K", "Qy", "Sz"):
        ref = _host_apply(box, form, x)
        got = op.apply(x, form).cpu().numpy()
        assert np.linalg.norm(got - ref) <= 1e-12 * np.linalg.norm(ref), form
    b = tb.poisson_rhs(box)
    dinv = 1.0 / box.diag_A()

    def host_pcg(tol):
        """the same Jacobi-PCG on the host with the sum-factorised apply"""
        xh = np.zeros_like(b)
        r = b.copy()
        z = dinv * r
        pv = z.copy()
        rz = r @ z
        its = 0
        for its in range(1, 20001):
            Ap = _host_apply(box, "A", pv)
            al = rz / (pv @ Ap)
            xh += al * pv
            r -= al * Ap
            if np.linalg.norm(r) <= tol * np.linalg.norm(b):
                break
            z = dinv * r
            rzn = r @ z
            pv = z + (rzn / rz) * pv
            rz = rzn
        return xh, its

    xs, rep = solve_spd(op, b, tol=1e-10, maxiter=20000)
    assert rep.success, rep
    _, its = host_pcg(1e-10)
    assert abs(its - rep.iterations) <= max(1, 0.02 * rep.iterations)
    # solutions compared at tol 1e-12: the ~950-iteration solves drift apart in
    # rounding by about 1e-8 at tol 1e-10 (different summation orders)
    xs, rep = solve_spd(op, b, tol=1e-12, maxiter=20000)
    assert rep.success, rep
    xh, _ = host_pcg(1e-12)
    assert np.linalg.norm(xs - xh) <= 1e-8 * np.linalg.norm(xh)
    op.close()
    torch.cuda.synchronize()
