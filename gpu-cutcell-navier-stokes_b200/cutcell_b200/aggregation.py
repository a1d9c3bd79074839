"""Polynomial-preserving aggregation (extension) ``E`` for 3D cut-cell spaces.

Same construction as ``polynomial_preserving_extension_3d``
(code/bell_3d_core.py:471-542): coordinates with fluid-mass ratio
``gamma >= 0.04`` are interior and map to themselves; every other active
coordinate gets the least-squares weights that reproduce all total-degree
``<= p`` monomials (spline coefficients by Greville interpolation,
code/bell_3d_core.py:444-458) from its nearest interior Greville neighbours,
starting from ``n_terms + 8`` and growing by 8 while the moment matrix is rank
deficient (``matrix_rank(tol=1e-10)``), at most ``6 n_terms``; weights with
``|w| <= 1e-14`` are dropped.  The neighbour ordering uses the same
``argsort`` of Euclidean Greville distances, evaluated in row chunks so the
distance matrix never has to be materialised whole (each row's ordering is
independent of the others, so chunking changes no index).

Besides the CSR matrix this module emits the device layout the gather/scatter
kernels consume: an int32 map ``red_of_full`` for the identity rows, a CSR of
the small rows, and the transposed CSR of the small rows (sorted by full
index) so ``E^T`` needs no atomics.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from .bspline import OpenUniformBasis, polynomial_coefficients


@dataclass
class Extension:
    E: sp.csr_matrix
    interior: np.ndarray
    small_support: np.ndarray
    active: np.ndarray
    gamma: np.ndarray
    polynomial_residual: float

    @property
    def n_full(self) -> int:
        return self.E.shape[0]

    @property
    def n_red(self) -> int:
        return self.E.shape[1]

    def device_layout(self) -> dict:
        """Index maps for the E gather / E^T scatter kernels (int32, fp64)."""
        n_full, n_red = self.E.shape
        red_of_full = np.full(n_full, -1, dtype=np.int32)
        red_of_full[self.interior] = np.arange(n_red, dtype=np.int32)
        small = np.asarray(self.small_support, dtype=np.int64)
        Es = self.E[small].tocsr()
        Es.sort_indices()
        small_slot = np.full(n_full, -1, dtype=np.int32)
        small_slot[small] = np.arange(small.size, dtype=np.int32)
        # transposed small rows: for reduced column j, entries (full row b, weight)
        EsT = sp.csr_matrix(
            (Es.data, Es.indices, Es.indptr), shape=(small.size, n_red)
        ).T.tocsr()
        EsT.sort_indices()
        return {
            "red_of_full": red_of_full,
            "full_of_red": np.asarray(self.interior, dtype=np.int32),
            "small_rows": small.astype(np.int32),
            "small_slot": small_slot,
            "small_ptr": Es.indptr.astype(np.int32),
            "small_idx": Es.indices.astype(np.int32),
            "small_val": Es.data.astype(np.float64),
            "smallT_ptr": EsT.indptr.astype(np.int32),
            # column of EsT is the slot in small_rows -> convert to full index
            "smallT_row": small[EsT.indices].astype(np.int32),
            "smallT_val": EsT.data.astype(np.float64),
        }


def greville_3d(basis: OpenUniformBasis) -> np.ndarray:
    g = basis.greville
    nb = basis.n_basis
    X = np.tile(np.tile(g, nb), nb)
    Y = np.tile(np.repeat(g, nb), nb)
    Z = np.repeat(g, nb * nb)
    return np.column_stack([X, Y, Z])


def monomial_rows_3d(basis: OpenUniformBasis, degree: int) -> np.ndarray:
    c = polynomial_coefficients(basis, degree)
    rows = []
    for total in range(degree + 1):
        for a in range(total + 1):
            for b in range(total - a + 1):
                cc = total - a - b
                rows.append(np.einsum("k,j,i->kji", c[cc], c[b], c[a]).reshape(-1))
    return np.vstack(rows)


def build_extension(
    gamma: np.ndarray,
    basis: OpenUniformBasis,
    degree: int,
    *,
    support_threshold: float = 0.04,
    preserve_degree: int | None = None,
    mass_diag: np.ndarray | None = None,
    chunk: int = 64,
    neighbour_search: str = "auto",
) -> Extension:
    """Polynomial-preserving extension (code/bell_3d_core.py:471-542).

    ``neighbour_search``: "dense" sorts all interior Greville distances per
    small DOF with NumPy's default argsort, as the reference does (bit-exact
    E, ties included).  "tree" takes the nearest candidates from a k-d tree
    (everything at or inside the needed radius, sorted by distance with ties
    in interior order): the same kind of polynomial-preserving extension,
    but equidistant neighbours at the cut-off may be chosen differently from
    the reference's unstable sort.  "auto" keeps the dense search up to
    5e8 small x interior distances (n <= 40 at p = 3) and uses the tree
    beyond, where the dense sort takes minutes."""
    deg = degree if preserve_degree is None else int(preserve_degree)
    gamma = np.asarray(gamma, dtype=float)
    active = np.where(gamma > 0.0)[0]
    interior = np.where(gamma >= support_threshold)[0]
    small = np.array([i for i in active if gamma[i] < support_threshold], dtype=int)
    if interior.size == 0:
        raise ValueError("no interior coordinates")
    n_full = gamma.size
    greville = greville_3d(basis)
    col = np.full(n_full, -1, dtype=np.int64)
    col[interior] = np.arange(interior.size)
    rows_t = [interior.astype(np.int64)]
    cols_t = [np.arange(interior.size, dtype=np.int64)]
    vals_t = [np.ones(interior.size)]

    if deg == 0:
        # constants only: mass-weighted average of the 8 nearest interior
        # neighbours (code/bell_3d_core.py:496-511)
        m_diag = np.asarray(mass_diag if mass_diag is not None else np.ones(n_full))
        for b in small:
            dist = np.linalg.norm(greville[interior] - greville[int(b)], axis=1)
            nb = interior[np.argsort(dist)[:8]]
            w = np.maximum(m_diag[nb], 0.0)
            w = w / max(float(w.sum()), 1.0e-300)
            rows_t.append(np.full(nb.size, int(b)))
            cols_t.append(col[nb])
            vals_t.append(w)
        E = sp.csr_matrix(
            (np.concatenate(vals_t), (np.concatenate(rows_t), np.concatenate(cols_t))),
            shape=(n_full, interior.size),
        )
        E.sort_indices()
        return Extension(E, interior, small, active, gamma, 0.0)

    poly = monomial_rows_3d(basis, deg)
    n_terms = poly.shape[0]
    gi = greville[interior]
    # only the first 6 n_terms + 8 neighbours are ever used (the rank loop below)
    need = 6 * n_terms + 8
    tree = None
    use_tree = neighbour_search == "tree" or (
        neighbour_search == "auto" and interior.size > 4 * need and small.size * interior.size > 5.0e8
    )
    if use_tree:
        from scipy.spatial import cKDTree

        tree = cKDTree(gi)

    def nearest_order(blk):
        """Per small DOF: interior positions by Greville distance, ties in
        interior order (the stable order of a full argsort), at least the
        first ``need`` of them."""
        if tree is None:
            return np.argsort(np.linalg.norm(gi[None, :, :] - greville[blk][:, None, :], axis=2), axis=1)
        out = []
        dk, _ = tree.query(greville[blk], k=need)
        for r, b in enumerate(blk):
            # every point at or inside the need-th distance, ties included
            cand = np.asarray(tree.query_ball_point(greville[int(b)], r=float(dk[r, -1]) * (1.0 + 1e-9) + 1e-300))
            cand.sort()
            dist = np.linalg.norm(gi[cand] - greville[int(b)], axis=1)
            out.append(cand[np.argsort(dist, kind="stable")])
        return out

    # The neighbour orders of the chunks are independent and NumPy releases the
    # GIL in the distance reductions and sorts, so they run on a thread pool;
    # every row is the same computation as the sequential loop (bit-identical E).
    import os
    from concurrent.futures import ThreadPoolExecutor

    blocks = [small[s0 : s0 + chunk] for s0 in range(0, small.size, chunk)]
    workers = max(1, min(8, os.cpu_count() or 1, len(blocks)))
    if tree is None and workers > 1:
        # a bound on the concurrent distance tables: chunk x interior x 4 doubles each
        workers = max(1, min(workers, int(2.0e9 // max(1, chunk * interior.size * 32))))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        orders = list(pool.map(nearest_order, blocks))
    for blk, order in zip(blocks, orders):
        for r, b in enumerate(blk):
            ordered = interior[order[r]]
            k = n_terms
            chosen = ordered[: k + 8]
            C = poly[:, chosen]
            while np.linalg.matrix_rank(C, tol=1.0e-10) < n_terms and len(chosen) < min(
                len(ordered), 6 * n_terms
            ):
                k += 8
                chosen = ordered[: k + 8]
                C = poly[:, chosen]
            w, *_ = np.linalg.lstsq(C, poly[:, int(b)], rcond=None)
            keep = np.abs(w) > 1.0e-14
            rows_t.append(np.full(int(keep.sum()), int(b)))
            cols_t.append(col[chosen[keep]])
            vals_t.append(w[keep])
    E = sp.csr_matrix(
        (np.concatenate(vals_t), (np.concatenate(rows_t), np.concatenate(cols_t))),
        shape=(n_full, interior.size),
    )
    E.sort_indices()
    active_mask = (gamma > 0.0).astype(float)
    res = 0.0
    for row in poly:
        res = max(res, float(np.max(np.abs(E @ row[interior] - row * active_mask))))
    return Extension(E, interior, small, active, gamma, res)


# ---- 1D and tensor-product aggregation (axis-aligned cut boxes) ----


def cut_interval_gamma(basis: OpenUniformBasis, left: float) -> np.ndarray:
    """gamma_i = int_left^1 N_i^2 / int_0^1 N_i^2 on the cut interval [left, 1]
    (the diagonal ratio of assemble_cut_matrices' H and H_background,
    code/cut_spline_sbp.py:90-146), by Gauss rules exact for N_i^2."""
    from .bspline import gauss_legendre01, local_values

    p, ne, h = basis.degree, basis.n_elements, basis.h
    xg, wg = gauss_legendre01(p + 1)
    cut = np.zeros(basis.n_basis)
    full = np.zeros(basis.n_basis)
    for e in range(ne):
        a, b = e * h, (e + 1) * h
        for lo, acc in ((a, full), (max(a, left), cut)):
            if b <= lo:
                continue
            x = lo + (b - lo) * xg
            N, _ = local_values(basis, np.full(x.size, e), x)
            acc[e : e + p + 1] += ((b - lo) * wg) @ (N * N)
    g = np.zeros_like(cut)
    pos = full > 0.0
    g[pos] = cut[pos] / full[pos]
    return g


def extension_1d(basis: OpenUniformBasis, left: float, support_threshold: float = 0.05,
                 preserve_degree: int | None = None, active_tol: float = 1.0e-25):
    """polynomial_preserving_extension on the cut interval [left, 1]
    (code/cut_spline_sbp.py:156-198): interior functions (gamma >= threshold)
    get identity columns; each small active function takes the least-squares
    weights that reproduce the monomials up to the degree from its nearest
    interior Greville neighbours (ties in interior order), the stencil grown
    from degree + 1 up to degree + 6 until the moment block has full rank.
    Returns (E dense (n_basis, n_red), interior, small, active, gamma, degree)."""
    from .bspline import polynomial_coefficients

    gamma = cut_interval_gamma(basis, left)
    active = np.where(gamma > active_tol)[0]
    interior = np.where(gamma >= support_threshold)[0]
    small = active[gamma[active] < support_threshold]
    if interior.size == 0:
        raise ValueError("no interior basis functions")
    deg = min(basis.degree if preserve_degree is None else preserve_degree, interior.size - 1)
    poly = polynomial_coefficients(basis, deg)
    col = np.full(basis.n_basis, -1, dtype=np.int64)
    col[interior] = np.arange(interior.size)
    E = np.zeros((basis.n_basis, interior.size))
    E[interior, np.arange(interior.size)] = 1.0
    g = basis.greville
    for i in small:
        ordered = interior[np.argsort(np.abs(g[interior] - g[i]), kind="stable")]
        chosen = ordered[: deg + 1]
        for k in range(deg + 1, min(ordered.size, deg + 6) + 1):
            if np.linalg.matrix_rank(poly[:, ordered[:k]], tol=1.0e-12) == deg + 1:
                chosen = ordered[:k]
                break
        w = np.linalg.lstsq(poly[:, chosen], poly[:, i], rcond=None)[0]
        E[i, col[chosen]] = w
    return E, interior, small, active, gamma, deg


def tensor_extension(basis: OpenUniformBasis, lefts, support_threshold: float = 0.05,
                     preserve_degree: int | None = None) -> Extension:
    """E = Ez (x) Ey (x) Ex of a cut box with low-side cuts at ``lefts``
    (assemble_cut_3d, code/cut_3d_sbp.py:89-146).  Reduced columns follow the
    Kronecker order (z slowest); DOFs are x-fastest."""
    parts = [extension_1d(basis, float(a), support_threshold, preserve_degree) for a in lefts]
    (Ex, ix, _, ax, gx, _), (Ey, iy, _, ay, gy, _), (Ez, iz, _, az, gz, _) = parts
    E = sp.kron(sp.csr_matrix(Ez), sp.kron(sp.csr_matrix(Ey), sp.csr_matrix(Ex))).tocsr()
    E.eliminate_zeros()
    E.sort_indices()
    nb = basis.n_basis
    lin = lambda sz, sy, sx: ((sz[:, None, None] * nb + sy[None, :, None]) * nb + sx[None, None, :]).ravel()
    interior = lin(iz, iy, ix)
    active = np.sort(lin(az, ay, ax))
    small = np.setdiff1d(active, interior)
    gamma = np.kron(gz, np.kron(gy, gx))
    return Extension(E, interior, small, active, gamma, 0.0)
