"""Matrix-free ``E^T A E`` on the device: tile layout (host) + C-ABI context.

``CutCellOperator`` is the structured entry of the solver boundary: it holds
the element-structured operator of a ``CutCellProblem`` and the aggregation
``Extension``, uploads them once, and applies / solves through
libcutcell_b200.so.  It replaces the explicit ``restrict_spd(A, E)`` product
(code/bell_3d_core.py:550-552) followed by a CSR Krylov loop
(code/fast_solver_backends.py:194-289).

Tile layout: the element grid is cut into ``tile^3`` element tiles.  A tile
whose elements are all uncut and inside the fluid is FULL and is applied as
one Kronecker sum of tile-assembled 1D factors (``(tile+p) x (tile+p)``); a
tile containing cut (or missing) elements is MIXED and applied element by
element; a tile with no fluid is EMPTY and skipped.
"""

from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp

from . import _lib
from .aggregation import Extension
from .problem import CUT, FULL, CutCellProblem

TILE_EMPTY, TILE_FULL, TILE_MIXED = 0, 1, 2


@dataclass
class TileLayout:
    tile: int
    n_tiles_axis: int
    tile_kind: np.ndarray  # (nta^3,) int32
    item_list: np.ndarray  # work items, >= 0 tile id, < 0 cut chunk -(k+1)
    tile_eptr: np.ndarray  # (nta^3 + 1,) uncut elements of mixed tiles
    tile_elem: np.ndarray
    TM: np.ndarray  # (nta, D, D)
    TA: np.ndarray
    TK: np.ndarray  # (3, nta, D, D)
    cut_chunk: int
    cut_base: np.ndarray  # (ncut,) first full DOF of each cut element
    cut_dof_slot: np.ndarray  # (n_full,)
    cut_dof_ptr: np.ndarray
    cut_dof_ent: np.ndarray  # cut * P + local row
    n_mixed: int = 0  # leading mixed tiles in item_list (block-level items; full tiles are warp-level)

    @property
    def tile_list(self) -> np.ndarray:
        return self.item_list[self.item_list >= 0]


def build_tile_layout(prob: CutCellProblem, tile: int = 4, cut_chunk: int = 2) -> TileLayout:
    n, p = prob.n_elements, prob.degree
    T = int(tile)
    nta = -(-n // T)
    D = T + p
    nb = n + p
    P = prob.P
    et = prob.elem_type
    kind = np.zeros(nta**3, dtype=np.int32)
    eptr = np.zeros(nta**3 + 1, dtype=np.int32)
    elems = []
    mixed_cost = {}
    for tz in range(nta):
        for ty in range(nta):
            for tx in range(nta):
                t = (tz * nta + ty) * nta + tx
                sub = et[tz * T : tz * T + T, ty * T : ty * T + T, tx * T : tx * T + T]
                complete = sub.shape == (T, T, T)
                if complete and np.all(sub == FULL):
                    kind[t] = TILE_FULL
                elif np.any(sub == FULL):
                    kind[t] = TILE_MIXED
                    lz, ly, lx = np.nonzero(sub == FULL)
                    elems.append(((lz * T + ly) * T + lx).astype(np.int32))
                    mixed_cost[t] = int(lx.size)
                eptr[t + 1] = eptr[t] + (elems[-1].size if kind[t] == TILE_MIXED else 0)
    tile_elem = np.concatenate(elems) if elems else np.zeros(0, np.int32)
    ncut = int(prob.cut_ids.size)
    nchunk = -(-ncut // cut_chunk)
    # work order: heaviest mixed tiles, then full tiles
    mixed = sorted(mixed_cost, key=lambda t: (-mixed_cost[t], t))
    full = [int(t) for t in np.nonzero(kind == TILE_FULL)[0]]
    # cut elements are claimed warp by warp after the tiles (not tile items)
    item_list = np.array(mixed + full, dtype=np.int32)
    # tile-assembled 1D factors
    TM = np.zeros((nta, D, D))
    TK = np.zeros((3, nta, D, D))
    for t in range(nta):
        for le in range(T):
            e = t * T + le
            if e >= n:
                break
            sl = slice(le, le + p + 1)
            TM[t, sl, sl] += prob.M1[e]
            for ax in range(3):
                TK[ax, t, sl, sl] += prob.Kt1[ax, e]
    TA = prob.a_mass * TM + TK[0]
    # cut elements: first DOF and the DOF -> (cut, local row) lists
    cz, cy, cx = np.unravel_index(prob.cut_ids, (n, n, n))
    cut_base = ((cz * nb + cy) * nb + cx).astype(np.int32)
    slot = np.full(prob.n_full, -1, dtype=np.int32)
    if ncut:
        R = prob.element_rows(cx, cy, cz)  # (ncut, P)
        g = R.ravel()
        ent = (np.arange(ncut)[:, None] * P + np.arange(P)[None, :]).ravel()
        order = np.lexsort((ent, g))
        g, ent = g[order], ent[order]
        uniq, start = np.unique(g, return_index=True)
        slot[uniq] = np.arange(uniq.size, dtype=np.int32)
        ptr = np.append(start, g.size).astype(np.int32)
        ent = ent.astype(np.int32)
    else:
        ptr = np.zeros(1, dtype=np.int32)
        ent = np.zeros(0, dtype=np.int32)
    return TileLayout(T, nta, kind, item_list, eptr, tile_elem, TM, TA, TK, cut_chunk, cut_base, slot, ptr, ent,
                      n_mixed=len(mixed))


def jacobi_diagonal(prob: CutCellProblem, ext: Extension) -> np.ndarray:
    """diag(E^T A E) from the element blocks, without forming E^T A E."""
    n, p = prob.n_elements, prob.degree
    n_red = ext.n_red
    lay = ext.device_layout()
    red_of_full = lay["red_of_full"]
    small_mask = np.zeros(prob.n_full, dtype=bool)
    small_mask[ext.small_support] = True
    diag = np.zeros(n_red)
    E = ext.E.tocsr()
    # full elements
    ez, ey, ex = np.nonzero(prob.elem_type == FULL)
    for s in range(0, ex.size, 8192):
        sl = slice(s, s + 8192)
        R = prob.element_rows(ex[sl], ey[sl], ez[sl])
        near = small_mask[R].any(axis=1)
        dM = np.einsum("eii->ei", prob.M1)
        dK = [np.einsum("eii->ei", prob.Kt1[a]) for a in range(3)]
        k3 = lambda a, b, c: (a[:, :, None, None] * b[:, None, :, None] * c[:, None, None, :]).reshape(a.shape[0], -1)
        exs, eys, ezs = ex[sl], ey[sl], ez[sl]
        dblk = (
            k3(dM[ezs], dM[eys], prob.a_mass * dM[exs] + dK[0][exs])
            + k3(dM[ezs], dK[1][eys], dM[exs])
            + k3(dK[2][ezs], dM[eys], dM[exs])
        )
        far = ~near
        cols = red_of_full[R[far]]
        ok = cols >= 0
        np.add.at(diag, cols[ok], dblk[far][ok])
        idx = np.nonzero(near)[0]
        if idx.size:
            blocks = prob.full_element_blocks(exs[idx], eys[idx], ezs[idx])
            for k, i in enumerate(idx):
                _near_block(diag, E, R[i], blocks[k])
    cz, cy, cx = np.unravel_index(prob.cut_ids, (n, n, n))
    if prob.cut_ids.size:
        R = prob.element_rows(cx, cy, cz)
        for k in range(prob.cut_ids.size):
            if small_mask[R[k]].any():
                _near_block(diag, E, R[k], prob.cut_mats[k])
            else:
                cols = red_of_full[R[k]]
                ok = cols >= 0
                np.add.at(diag, cols[ok], np.diag(prob.cut_mats[k])[ok])
    return diag


def _near_block(diag, E, rows, A):
    Ee = E[rows]
    cols = np.unique(Ee.indices)
    if cols.size == 0:
        return
    Ed = Ee[:, cols].toarray()
    diag[cols] += np.einsum("aj,ab,bj->j", Ed, A, Ed)


def _dev(x, dtype, device):
    import torch

    return torch.as_tensor(np.ascontiguousarray(x)).to(device=device, dtype=dtype)


class CutCellOperator:
    """Device-resident matrix-free ``E^T A E`` with PCG/IR solves."""

    def __init__(self, prob: CutCellProblem, ext: Extension, *, tile: int = 4, device="cuda", diag=None):
        import torch

        lib = _lib.load()
        self.problem = prob
        self.extension = ext
        self.n = ext.n_red
        self.shape = (ext.n_red, ext.n_red)
        self.device = torch.device(device)
        lay = build_tile_layout(prob, tile)
        self.layout = lay
        el = ext.device_layout()
        if diag is None:
            diag = jacobi_diagonal(prob, ext)
        self.diag = np.asarray(diag, dtype=float)
        i32, f64 = torch.int32, torch.float64
        dv = self.device
        P = prob.P
        t = {}
        t["item_list"] = _dev(lay.item_list, i32, dv)
        t["tile_kind"] = _dev(lay.tile_kind, i32, dv)
        t["tile_eptr"] = _dev(lay.tile_eptr, i32, dv)
        t["tile_elem"] = _dev(np.append(lay.tile_elem, 0), i32, dv)
        t["tile_ecut"] = t["tile_elem"]
        t["cut_base"] = _dev(np.append(lay.cut_base, 0), i32, dv)
        t["cut_dof_slot"] = _dev(lay.cut_dof_slot, i32, dv)
        t["cut_dof_ptr"] = _dev(lay.cut_dof_ptr, i32, dv)
        t["cut_dof_ent"] = _dev(np.append(lay.cut_dof_ent, 0), i32, dv)
        need = np.union1d(np.asarray(ext.interior), np.asarray(ext.small_support)).astype(np.int32)
        t["need"] = _dev(need, i32, dv)
        t["M1"] = _dev(prob.M1, f64, dv)
        t["Kt1"] = _dev(prob.Kt1, f64, dv)
        t["TM"] = _dev(lay.TM, f64, dv)
        t["TA"] = _dev(lay.TA, f64, dv)
        t["TK"] = _dev(lay.TK, f64, dv)
        t["cut_mats"] = _dev(prob.cut_mats.reshape(-1, P * P) if prob.cut_ids.size else np.zeros((1, P * P)), f64, dv)
        for k in ("red_of_full", "small_slot", "small_ptr", "full_of_red", "smallT_ptr"):
            t[k] = _dev(el[k], i32, dv)
        for k in ("small_idx", "smallT_row"):
            t[k] = _dev(np.append(el[k], 0), i32, dv)
        for k in ("small_val", "smallT_val"):
            t[k] = _dev(np.append(el[k], 0.0), f64, dv)
        t["diag"] = _dev(self.diag, f64, dv)
        self._t = t
        desc = _lib.CutcellTileDesc()
        desc.n_elements = prob.n_elements
        desc.degree = prob.degree
        desc.tile = lay.tile
        desc.n_tiles_axis = lay.n_tiles_axis
        desc.n_items = int(lay.item_list.size)
        desc.n_mixed = int(lay.n_mixed)
        desc.cut_chunk = int(lay.cut_chunk)
        desc.n_cut = int(prob.cut_ids.size)
        desc.n_full = prob.n_full
        desc.n_red = ext.n_red
        desc.n_small = int(ext.small_support.size)
        desc.n_need = int(need.size)
        desc.a_mass = prob.a_mass
        for name, _ in _lib.CutcellTileDesc._fields_:
            if name in t:
                setattr(desc, name, t[name].data_ptr())
        self._desc = desc
        ctx = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(lib.cutcell_pcg_create_tiles(C.byref(desc), C.byref(ctx)), "cutcell_pcg_create_tiles")
        self._ctx = ctx
        self._lib = lib

    # -- helpers -----------------------------------------------------------
    def reduced_load(self) -> np.ndarray:
        return np.asarray(self.extension.E.T @ self.problem.load)

    def set_refinement(self, replace_factor: float = 0.1, max_replacements: int = 200) -> None:
        """Controls of the FP32 / BF16 forms (PCG with the reduced-precision
        operator and FP64 residual replacement): the recursive residual is
        replaced by the FP64 true residual each time its norm falls by
        ``replace_factor``; at most ``max_replacements`` replacements."""
        _lib.check(
            self._lib.cutcell_set_refinement(self._ctx, float(replace_factor), 0, int(max_replacements)),
            "cutcell_set_refinement",
        )

    def apply(self, x, precision: str = "fp64"):
        import torch

        x = torch.as_tensor(x, dtype=torch.float64, device=self.device).contiguous()
        y = torch.empty_like(x)
        _lib.check(
            self._lib.cutcell_apply(self._ctx, x.data_ptr(), y.data_ptr(), _lib.PRECISIONS[precision], _lib.current_stream_ptr()),
            "cutcell_apply",
        )
        return y

    def gather(self, x_red):
        import torch

        x_red = torch.as_tensor(x_red, dtype=torch.float64, device=self.device).contiguous()
        out = torch.empty(self.problem.n_full, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.cutcell_ext_gather(self._ctx, x_red.data_ptr(), out.data_ptr(), _lib.current_stream_ptr()), "gather")
        return out

    def scatter(self, y_full):
        import torch

        y_full = torch.as_tensor(y_full, dtype=torch.float64, device=self.device).contiguous()
        out = torch.empty(self.n, dtype=torch.float64, device=self.device)
        _lib.check(self._lib.cutcell_ext_scatter(self._ctx, y_full.data_ptr(), out.data_ptr(), _lib.current_stream_ptr()), "scatter")
        return out

    def solve_device(self, b, x=None, *, tol=1e-8, maxiter=5000, precision="fp64", preconditioner="jacobi"):
        """Solve with device-resident b / x (torch tensors); returns (x, CutcellReport)."""
        import torch

        b = torch.as_tensor(b, dtype=torch.float64, device=self.device).contiguous()
        if x is None:
            x = torch.empty_like(b)
        rep = _lib.CutcellReport()
        pc = {"none": _lib.PRECOND_NONE, "jacobi": _lib.PRECOND_JACOBI, "jacobi+learned": _lib.PRECOND_JACOBI_LEARNED,
              "block": _lib.PRECOND_BLOCK, "twolevel": _lib.PRECOND_TWOLEVEL}[preconditioner]
        _lib.check(
            self._lib.cutcell_pcg_solve(
                self._ctx, b.data_ptr(), x.data_ptr(), float(tol), int(maxiter), _lib.PRECISIONS[precision], pc,
                C.byref(rep), _lib.current_stream_ptr(),
            ),
            "cutcell_pcg_solve",
        )
        return x, rep

    def close(self) -> None:
        if getattr(self, "_ctx", None):
            self._lib.cutcell_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
