"""Host-side setup of the product (basis, cut quadrature, element blocks, E,
tile layout) against the oracle and the reference's golden vectors."""

import numpy as np
import pytest
import scipy.sparse as sp

from cutcell_b200.aggregation import build_extension
from cutcell_b200.bspline import element_matrices_1d, global_values, make_basis
from cutcell_b200.cutgeom import PlaneLevelSet, cut_cell_quadrature
from cutcell_b200.operator import TILE_EMPTY, TILE_FULL, TILE_MIXED, build_tile_layout, jacobi_diagonal
from cutcell_b200.problem import FULL, _tensor_local, build_problem
from oracle import aggregation as oa
from oracle import assembly as oasm

from _systems import plane5, sphere, system


@pytest.mark.parametrize("n,p", [(5, 3), (8, 2), (6, 4), (3, 5)])
def test_basis_against_scipy(n, p):
    x = np.linspace(0, 1, 97)
    V = global_values(make_basis(n, p), x)
    np.testing.assert_allclose(V, oa.basis_matrix(n, p, x).T, atol=1e-14)


@pytest.mark.parametrize("n,p", [(6, 3), (4, 2), (5, 5)])
def test_1d_element_forms_against_oracle(n, p):
    M, K = element_matrices_1d(make_basis(n, p))
    Mo, Ko = oasm.interval_forms(n, p)
    np.testing.assert_allclose(M, Mo, atol=1e-15)
    np.testing.assert_allclose(K, Ko, rtol=1e-13, atol=1e-12)


@pytest.mark.parametrize("case", [0, 1, 2, 3])
def test_axis_cut_box_against_reference_1d_forms(golden, case):
    """A plane x = a cut must give H = Hz (x) Hy (x) Hx(a) with the reference's
    1D cut forms (code/cut_spline_sbp.py:90-129, code/cut_3d_sbp.py:112-113)."""
    g = np.load(golden / "cut1d.npz")
    n, p, frac = g[f"c{case}_meta"]
    n, p = int(n), int(p)
    if frac == 0.0:
        pytest.skip("uncut axis")
    a = frac / n
    c0 = [k for k in range(int(g["count"])) if tuple(g[f"c{k}_meta"][:2]) == (n, p) and g[f"c{k}_meta"][2] == 0.0]
    H0 = g[f"c{c0[0]}_H"] if c0 else oasm.interval_forms(n, p)[0]
    if not c0:
        H0 = None
    prob = build_problem(PlaneLevelSet((1.0, 0.0, 0.0), a), n, p, a_mass=1.0, a_stiff=0.0, nitsche=False)
    A = oasm.assemble_full(prob).toarray()
    Hx = g[f"c{case}_H"]
    if H0 is None:
        b = make_basis(n, p)
        M, _ = element_matrices_1d(b)
        H0 = np.zeros((n + p, n + p))
        for e in range(n):
            H0[e : e + p + 1, e : e + p + 1] += M[e]
    ref = np.kron(np.kron(H0, H0), Hx)
    np.testing.assert_allclose(A, ref, atol=1e-15 * n**3, rtol=0)
    # stiffness
    prob = build_problem(PlaneLevelSet((1.0, 0.0, 0.0), a), n, p, a_mass=0.0, a_stiff=1.0, nitsche=False)
    A = oasm.assemble_full(prob).toarray()
    K0 = np.zeros_like(H0)
    _, Kf = element_matrices_1d(make_basis(n, p))
    for e in range(n):
        K0[e : e + p + 1, e : e + p + 1] += Kf[e]
    Kx = g[f"c{case}_K"]
    ref = np.kron(np.kron(H0, H0), Kx) + np.kron(np.kron(H0, K0), Hx) + np.kron(np.kron(K0, H0), Hx)
    np.testing.assert_allclose(A, ref, atol=1e-12 * np.abs(ref).max(), rtol=0)


@pytest.mark.parametrize("phi", [plane5(), sphere()])
def test_cut_cell_green_identity(phi):
    """Q + Q^T = S on every cut cell (all faces), to round-off, with q = 3p+1
    (the 3D analogue of green_residuals_3d, code/cut_3d_sbp.py:149-154)."""
    n, p = 6, 2
    b = make_basis(n, p)
    h = b.h
    worst = 0.0
    for ex, ey, ez in [(1, 2, 3), (2, 2, 1), (1, 1, 1), (4, 2, 2), (0, 3, 3)]:
        cq = cut_cell_quadrature(phi, np.array([ex, ey, ez]) * h, h, 3 * p + 1, box_faces=False, cell_faces=True)
        if cq.wv.size == 0:
            continue
        pv, gv = _tensor_local(b, ex, ey, ez, cq.xv)
        ps, _ = _tensor_local(b, ex, ey, ez, cq.xs)
        for d in range(3):
            Q = (pv * cq.wv[:, None]).T @ gv[d]
            S = (ps * (cq.ws * cq.ns[:, d])[:, None]).T @ ps
            worst = max(worst, np.abs(Q + Q.T - S).max())
    assert worst < 1e-14


def test_plane_cut_volume_exact():
    phi = plane5(0.23)
    prob = build_problem(phi, 6, 2)
    nvec = np.array([np.cos(np.deg2rad(5)), np.sin(np.deg2rad(5)), 0.0])
    # volume of {n.x >= 0.23} in the unit cube: integrate over y analytically
    ys = np.linspace(0, 1, 200001)
    xcut = np.clip((0.23 - nvec[1] * ys) / nvec[0], 0, 1)
    exact = np.trapezoid(1.0 - xcut, ys)
    assert abs(prob.cut_fractions.sum() / 216.0 - exact) < 1e-9


@pytest.mark.parametrize("name", ["ext3d_sphere", "ext3d_bell"])
def test_product_extension_bit_exact(golden, name):
    g = np.load(golden / f"{name}.npz")
    Eref = sp.csr_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"]))
    ext = build_extension(g["gamma"], make_basis(int(g["n"]), int(g["p"])), int(g["p"]))
    assert np.array_equal(ext.E.indptr, Eref.indptr) and np.array_equal(ext.E.indices, Eref.indices)
    assert abs(ext.E - Eref).max() <= 1e-12
    assert ext.polynomial_residual < 1e-9


def test_device_layout_reproduces_E():
    g_prob, ext, *_ = system("sphere", 6, 2)
    lay = ext.device_layout()
    rng = np.random.default_rng(0)
    x = rng.standard_normal(ext.n_red)
    xf = np.zeros(ext.n_full)
    for i in range(ext.n_full):
        r = lay["red_of_full"][i]
        if r >= 0:
            xf[i] = x[r]
        elif lay["small_slot"][i] >= 0:
            s = lay["small_slot"][i]
            k0, k1 = lay["small_ptr"][s], lay["small_ptr"][s + 1]
            xf[i] = lay["small_val"][k0:k1] @ x[lay["small_idx"][k0:k1]]
    np.testing.assert_allclose(xf, ext.E @ x, rtol=1e-14, atol=1e-14)
    y = rng.standard_normal(ext.n_full)
    yr = y[lay["full_of_red"]].copy()
    for j in range(ext.n_red):
        k0, k1 = lay["smallT_ptr"][j], lay["smallT_ptr"][j + 1]
        yr[j] += lay["smallT_val"][k0:k1] @ y[lay["smallT_row"][k0:k1]]
    np.testing.assert_allclose(yr, ext.E.T @ y, rtol=1e-13, atol=1e-13)


@pytest.mark.parametrize("kind,n,p", [("sphere", 6, 2), ("plane", 6, 3), ("sphere", 9, 3)])
def test_tile_layout_reproduces_operator(kind, n, p):
    """Host emulation of the device work items (full tiles, uncut elements of
    mixed tiles, cut-element chunks + the DOF -> cut lists) equals E^T A E."""
    prob, ext, A_full, A_red, b = system(kind, n, p)
    lay = build_tile_layout(prob, 4)
    T, nta, D = lay.tile, lay.n_tiles_axis, lay.tile + p
    nb = n + p
    P = prob.P
    rng = np.random.default_rng(1)
    x = rng.standard_normal(ext.n_red)
    xf = ext.E @ x
    yf = np.zeros(ext.n_full)
    seen = np.zeros((n, n, n), dtype=int)
    ycut = np.zeros((prob.cut_ids.size, P))
    for c in range(prob.cut_ids.size):
        base = lay.cut_base[c]
        ez, ey, ex = np.unravel_index(prob.cut_ids[c], (n, n, n))
        assert base == (ez * nb + ey) * nb + ex
        R = prob.element_rows(ex, ey, ez)[0]
        ycut[c] = prob.cut_mats[c] @ xf[R]
        seen[ez, ey, ex] += 1
    for code in lay.item_list:
        if code < 0:
            k = -code - 1
            for c in range(k * lay.cut_chunk, min((k + 1) * lay.cut_chunk, prob.cut_ids.size)):
                base = lay.cut_base[c]
                ez, ey, ex = np.unravel_index(prob.cut_ids[c], (n, n, n))
                assert base == (ez * nb + ey) * nb + ex
                R = prob.element_rows(ex, ey, ez)[0]
                ycut[c] = prob.cut_mats[c] @ xf[R]
                seen[ez, ey, ex] += 1
            continue
        t = code
        tz, ty, tx = t // (nta * nta), (t // nta) % nta, t % nta
        if lay.tile_kind[t] == TILE_FULL:
            g = [np.arange(tt * T, tt * T + D) for tt in (tx, ty, tz)]
            rows = ((g[2][:, None] * nb + g[1][None, :])[:, :, None] * nb + g[0][None, None, :]).reshape(-1)
            B = (
                np.kron(np.kron(lay.TM[tz], lay.TM[ty]), lay.TA[tx])
                + np.kron(np.kron(lay.TM[tz], lay.TK[1, ty]), lay.TM[tx])
                + np.kron(np.kron(lay.TK[2, tz], lay.TM[ty]), lay.TM[tx])
            )
            yf[rows] += B @ xf[rows]
            seen[tz * T : tz * T + T, ty * T : ty * T + T, tx * T : tx * T + T] += 1
        else:
            assert lay.tile_kind[t] == TILE_MIXED
            for it in range(lay.tile_eptr[t], lay.tile_eptr[t + 1]):
                le = lay.tile_elem[it]
                lx, ly, lz = le % T, (le // T) % T, le // (T * T)
                ex, ey, ez = tx * T + lx, ty * T + ly, tz * T + lz
                assert prob.elem_type[ez, ey, ex] == FULL
                R = prob.element_rows(ex, ey, ez)[0]
                B = prob.full_element_blocks(np.array([ex]), np.array([ey]), np.array([ez]))[0]
                yf[R] += B @ xf[R]
                seen[ez, ey, ex] += 1
    assert np.array_equal(seen, (prob.elem_type != 0).astype(int))
    # cut partials through the DOF -> cut lists
    for g in np.nonzero(lay.cut_dof_slot >= 0)[0]:
        s_ = lay.cut_dof_slot[g]
        for e in lay.cut_dof_ent[lay.cut_dof_ptr[s_] : lay.cut_dof_ptr[s_ + 1]]:
            yf[g] += ycut[e // P, e % P]
    y = ext.E.T @ yf
    ref = A_red @ x
    np.testing.assert_allclose(y, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("kind,n,p", [("sphere", 6, 2), ("plane", 6, 3)])
def test_jacobi_diagonal(kind, n, p):
    prob, ext, A_full, A_red, b = system(kind, n, p)
    d = jacobi_diagonal(prob, ext)
    np.testing.assert_allclose(d, A_red.diagonal(), rtol=1e-12)


@pytest.mark.parametrize("kind", ["sphere", "plane"])
def test_native_setup_matches_python(kind):
    from cutcell_b200.problem import _setup_lib, manufactured_sine

    assert _setup_lib() is not None, "libcutcell_setup.so not built"
    u, f = manufactured_sine()
    phi = sphere() if kind == "sphere" else plane5()
    a = build_problem(phi, 6, 3, forcing=f, dirichlet=u, native=False)
    b = build_problem(phi, 6, 3, forcing=f, dirichlet=u, native=True)
    assert np.array_equal(a.cut_ids, b.cut_ids)
    np.testing.assert_allclose(b.cut_mats, a.cut_mats, rtol=0, atol=1e-13 * np.abs(a.cut_mats).max())
    np.testing.assert_allclose(b.load, a.load, rtol=0, atol=1e-13 * np.abs(a.load).max())
    np.testing.assert_allclose(b.gamma, a.gamma, rtol=0, atol=1e-13)
    np.testing.assert_allclose(b.cut_fractions, a.cut_fractions, rtol=0, atol=1e-14)


def test_extension_tree_search_is_a_valid_extension():
    """The k-d tree neighbour search (used for large grids) gives the same
    index sets and identity rows as the reference-ordered search and a
    polynomial-preserving E; only the choice among equidistant neighbours
    at the cut-off may differ."""
    from cutcell_b200.aggregation import build_extension
    from cutcell_b200.workloads import sphere_poisson

    prob, _ = sphere_poisson(16, 3, 0.31)
    a = build_extension(prob.gamma, prob.basis, 3, neighbour_search="dense")
    b = build_extension(prob.gamma, prob.basis, 3, neighbour_search="tree")
    for f in ("interior", "small_support", "active"):
        assert np.array_equal(getattr(a, f), getattr(b, f))
    rows = a.interior
    assert (a.E[rows] != b.E[rows]).nnz == 0
    assert b.polynomial_residual < 1e-11


def test_sliver_plane_worst_fraction_and_cube_volume():
    """Closed-form cube volume under a plane, and the sliver plane's worst
    cut cell against the product's cut quadrature."""
    from cutcell_b200.problem import build_problem
    from cutcell_b200.workloads import cube_volume_below, sliver_plane

    nrm = np.array([0.3, 0.5, 0.81])
    nrm /= np.linalg.norm(nrm)
    assert abs(cube_volume_below(nrm, nrm.sum())) - 1.0 < 1e-14 and cube_volume_below(nrm, 0.0) == 0.0
    # midpoint symmetry: the plane through the centre halves the cube
    assert abs(cube_volume_below(nrm, 0.5 * nrm.sum()) - 0.5) < 1e-14
    for eps in (1e-4, 0.05):
        phi = sliver_plane(8, [1.0, 2.0, 0.7], eps)
        prob = build_problem(phi, 8, 3)
        assert abs(prob.min_cut_fraction / eps - 1.0) < 1e-8


def test_plane_poisson_converges_at_optimal_order():
    """The plane-cut Poisson problem (normal rotated 5 degrees, worst cut cell
    0.15, p = 3) solved directly: L2 / H1 errors against u = sin sin sin,
    measured as solve_poisson_3d reports them (code/cut_3d_sbp.py:506-531),
    fall at the B-spline orders p + 1 and p."""
    import scipy.sparse.linalg as spla

    from cutcell_b200.cutgeom import PlaneLevelSet
    from cutcell_b200.problem import manufactured_sine, manufactured_sine_grad, solution_errors
    from cutcell_b200.workloads import plane_poisson
    from oracle.aggregation import restrict_spd

    u, _ = manufactured_sine()
    g = manufactured_sine_grad()
    errs = []
    for n in (4, 8):
        prob, ext, c = plane_poisson(n)
        assert abs(prob.min_cut_fraction - 0.15) < 1e-9
        a = np.deg2rad(5.0)
        phi = PlaneLevelSet((np.cos(a), np.sin(a), 0.0), c)
        A = restrict_spd(prob.assemble_full_csr(), ext.E)
        x = spla.spsolve(A.tocsc(), np.asarray(ext.E.T @ prob.load))
        errs.append(solution_errors(prob, phi, ext.E @ x, u, g))
    assert np.log2(errs[0]["l2"] / errs[1]["l2"]) > 3.5  # p + 1 = 4
    assert np.log2(errs[0]["h1"] / errs[1]["h1"]) > 2.7  # p = 3
    assert errs[1]["l2"] < 1e-4 and errs[1]["h1"] < 1e-3


def test_tensor_aggregation_matches_reference(golden):
    """1D polynomial-preserving extension and the tensor E of a cut box
    against the reference's own (tests/golden/tensor_ext.npz)."""
    from cutcell_b200.aggregation import extension_1d, tensor_extension
    from cutcell_b200.bspline import make_basis

    z = np.load(golden / "tensor_ext.npz")
    for k in range(int(z["count"])):
        n, p, frac = z[f"c{k}_meta"]
        b = make_basis(int(n), int(p))
        E, interior, small, active, gamma, deg = extension_1d(b, b.h * frac)
        np.testing.assert_array_equal(interior, z[f"c{k}_interior"])
        np.testing.assert_allclose(gamma, z[f"c{k}_gamma"], rtol=1e-12, atol=1e-16)
        assert E.shape == z[f"c{k}_E"].shape
        assert np.abs(E - z[f"c{k}_E"]).max() < 1e-10
    n, p = (int(v) for v in z["box_meta"][:2])
    fr = z["box_meta"][2:]
    b = make_basis(n, p)
    ext = tensor_extension(b, [b.h * f for f in fr])
    Eref = z["box_E"]
    assert ext.E.shape == Eref.shape
    assert np.abs(ext.E.toarray() - Eref).max() < 1e-10
    # the device layout accepts it: identity rows are the interior DOFs
    lay = ext.device_layout()
    assert np.array_equal(lay["full_of_red"], ext.interior)
