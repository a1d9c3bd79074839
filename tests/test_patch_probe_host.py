"""Patch-block probing (no GPU): the product's ``patch_blocks`` run against
an operator whose apply is the oracle's assembled E^T A E returns every
64x64 patch block exactly, for every tiling of the two-level form.

The patches probed together (one colour) must not be coupled by E^T A E.
The 8 parity colours alone are not enough next to cut cells, where the
extension rows of E couple same-parity patches: that probing mixed 33 of the
182 blocks of the sphere-cut n = 8, p = 3 system, and 252 of the sliver case
cut19's (p = 4, n = 16), 47 of them indefinite, so that the two-level solve
diverged there.  ``patch_colours`` separates every coupled pair."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from cutcell_b200.learned import DevicePatches, patch_blocks, patch_colours, patch_coupling, patch_layout


class _AssembledOp:
    """The attributes patch probing reads, with the assembled matrix as apply."""

    def __init__(self, prob, ext, A):
        self.problem, self.extension, self.A = prob, ext, A
        self.device = torch.device("cpu")
        self.n = ext.n_red

    def apply(self, v):
        return torch.as_tensor(self.A @ v.numpy())


def _sphere(n, p):
    from cutcell_b200.workloads import sphere_poisson

    return sphere_poisson(n, p, 0.31)


def _sliver(k):
    from cutcell_b200.aggregation import build_extension
    from cutcell_b200.problem import build_problem
    from cutcell_b200.workloads import sliver_plane, sliver_stress_cases

    nrm, eps = sliver_stress_cases(25)[k]
    prob = build_problem(sliver_plane(16, nrm, eps), 16, 4)
    return prob, build_extension(prob.gamma, prob.basis, 4)


@pytest.mark.parametrize("n,p", [(8, 3), (16, 3), (8, 4)])
def test_probe_colours_separate_coupled_patches(n, p):
    prob, ext = _sphere(n, p)
    op = _AssembledOp(prob, ext, None)
    for shift in (0, 1, 2, 3):
        lay = patch_layout(op, shift)
        colour = patch_colours(op, lay)
        K = patch_coupling(op, lay).tocoo()
        off = K.row != K.col
        assert not np.any(colour[K.row[off]] == colour[K.col[off]])


@pytest.mark.parametrize(
    "case,shifts",
    [("sphere n=8 p=3", (0, 1, 2, 3)), ("sphere n=8 p=4", (0, 1, 2, 3)), ("sliver cut19", (0,))],
)
def test_probed_patch_blocks_are_exact(case, shifts):
    from oracle.aggregation import restrict_spd
    from oracle.assembly import assemble_full

    prob, ext = _sliver(19) if case.startswith("sliver") else _sphere(8, int(case[-1]))
    A = restrict_spd(assemble_full(prob), ext.E).tocsr()
    op = _AssembledOp(prob, ext, A)
    for shift in shifts:
        lay = patch_layout(op, shift)
        blocks = patch_blocks(op, DevicePatches(op, lay))
        for k, row in enumerate(lay.red):
            m = row >= 0
            g = row[m]
            np.testing.assert_array_equal(blocks[k][np.ix_(m, m)], A[g][:, g].toarray())
            assert not np.any(blocks[k][~m]) and not np.any(blocks[k][:, ~m])
