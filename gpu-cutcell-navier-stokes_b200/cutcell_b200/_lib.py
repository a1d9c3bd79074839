"""ctypes binding of libcutcell_b200.so (the C ABI declared in include/cutcell_b200.h).

The library is built in-tree by ``cutcell_b200.build`` (nvcc, sm_100a).  There
is no fallback: if the shared object is missing or cannot be loaded, every
entry point raises ``CutcellLibraryError``.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_NAME = "libcutcell_b200.so"
LIB_PATH = Path(__file__).resolve().parent / LIB_NAME

OK = 0
E_NOCONV = 1
E_BREAKDOWN = 2
E_NAN = 3
E_SHAPE = 4
E_CUDA = 5
E_BARRIER = 6
E_ARG = 7

FP64 = 0
FP32_IR = 1
BF16_IR = 2
PRECISIONS = {"fp64": FP64, "fp32-ir": FP32_IR, "bf16-ir": BF16_IR}

PRECOND_NONE = 0
PRECOND_JACOBI = 1
PRECOND_JACOBI_LEARNED = 2
PRECOND_BLOCK = 3
PRECOND_TWOLEVEL = 4
MLP_NPARAM = 16576
MLP_IN, MLP_H, MLP_OUT = 128, 64, 64


class CutcellLibraryError(RuntimeError):
    pass


class CutcellReport(C.Structure):
    _fields_ = [
        ("status", C.c_int32),
        ("iterations", C.c_int32),
        ("outer_iterations", C.c_int32),
        ("blocks", C.c_int32),
        ("relative_residual", C.c_double),
        ("true_relative_residual", C.c_double),
        ("elapsed_ms", C.c_double),
    ]


_P = C.c_void_p


class CutcellTileDesc(C.Structure):
    _fields_ = [
        ("n_elements", C.c_int32),
        ("degree", C.c_int32),
        ("tile", C.c_int32),
        ("n_tiles_axis", C.c_int32),
        ("n_items", C.c_int32),
        ("cut_chunk", C.c_int32),
        ("n_cut", C.c_int32),
        ("n_full", C.c_int32),
        ("n_red", C.c_int32),
        ("n_small", C.c_int32),
        ("n_need", C.c_int32),
        ("a_mass", C.c_double),
        ("item_list", _P),
        ("tile_kind", _P),
        ("tile_eptr", _P),
        ("tile_elem", _P),
        ("tile_ecut", _P),
        ("M1", _P),
        ("Kt1", _P),
        ("TM", _P),
        ("TA", _P),
        ("TK", _P),
        ("cut_mats", _P),
        ("cut_base", _P),
        ("cut_dof_slot", _P),
        ("cut_dof_ptr", _P),
        ("cut_dof_ent", _P),
        ("need", _P),
        ("red_of_full", _P),
        ("small_slot", _P),
        ("small_ptr", _P),
        ("small_idx", _P),
        ("small_val", _P),
        ("full_of_red", _P),
        ("smallT_ptr", _P),
        ("smallT_row", _P),
        ("smallT_val", _P),
        ("diag", _P),
        ("n_mixed", C.c_int32),
    ]


class CutcellHillDesc(C.Structure):
    _fields_ = [(f, C.c_int32) for f in ("nr", "nz", "qpe", "nzb", "n_seg", "lmax", "n_part", "n2q")] + [
        (f, _P)
        for f in (
            "seg_q0", "seg_q1", "seg_pat", "seg_len", "pat_idx", "sp_ptr", "phi", "dpx", "dpy", "w2", "zb", "Vl",
            "dVl", "wzl", "g_ptr", "g_ent", "Mzinv", "M2inv",
        )
    ]


class CutcellCoarseDesc(C.Structure):
    _fields_ = [(f, C.c_int32) for f in ("nb", "nbc", "pw", "rw")] + [
        (f, _P) for f in ("plo", "pval", "rlo", "rval", "minv")
    ]


class CutcellBatchConfig(C.Structure):
    _fields_ = [
        ("cluster", C.c_int32),
        ("threads", C.c_int32),
        ("smem_matrix", C.c_int32),
        ("teams", C.c_int32),
    ]


# name -> (restype, argtypes); every symbol declared in include/cutcell_b200.h
SIGNATURES = {
    "cutcell_pcg_create_csr": (C.c_int, [C.c_int32, C.c_int32, _P, _P, _P, C.POINTER(_P)]),
    "cutcell_pcg_create_tiles": (C.c_int, [C.POINTER(CutcellTileDesc), C.POINTER(_P)]),
    "cutcell_set_refinement": (C.c_int, [_P, C.c_double, C.c_int32, C.c_int32]),
    "cutcell_pcg_solve": (
        C.c_int,
        [_P, _P, _P, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.POINTER(CutcellReport), _P],
    ),
    "cutcell_apply": (C.c_int, [_P, _P, _P, C.c_int32, _P]),
    "cutcell_ext_gather": (C.c_int, [_P, _P, _P, _P]),
    "cutcell_ext_scatter": (C.c_int, [_P, _P, _P, _P]),
    "cutcell_destroy": (C.c_int, [_P]),
    "cutcell_mlp_create": (C.c_int, [_P, C.c_int32, C.POINTER(_P)]),
    "cutcell_mlp_params": (C.c_int, [_P, _P, _P]),
    "cutcell_mlp_forward": (C.c_int, [_P, _P, C.c_int32, _P, _P]),
    "cutcell_mlp_train_step": (C.c_int, [_P, _P, _P, C.c_int32, C.c_float, _P, _P]),
    "cutcell_mlp_destroy": (C.c_int, [_P]),
    "cutcell_patch_features": (C.c_int, [_P, _P, _P, C.c_int32, _P, _P, _P, _P]),
    "cutcell_patch_targets": (C.c_int, [_P, _P, C.c_int32, _P, _P, _P, _P, _P]),
    "cutcell_pcg_set_learned": (C.c_int, [_P, _P, _P, _P, C.c_int32]),
    "cutcell_pcg_set_block_inverses": (C.c_int, [_P, _P]),
    "cutcell_pcg_set_patch_blocks": (C.c_int, [_P, _P, C.c_int32, _P, _P]),
    "cutcell_pcg_set_coarse": (C.c_int, [_P, _P]),
    "cutcell_pcg_set_twolevel_blocks": (C.c_int, [_P, _P, C.c_int32, _P, _P, _P, C.c_double]),
    "cutcell_fastdiag_create": (C.c_int, [C.c_int32, C.c_int32, _P, _P, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    "cutcell_fastdiag_solve": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P]),
    "cutcell_fastdiag_destroy": (C.c_int, [_P]),
    "cutcell_dgemm_nt": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _P, C.c_int64, C.c_int64, _P, C.c_int64, C.c_int64,
                                   _P, C.c_int64, C.c_double, _P, C.c_int64, C.c_int64, C.c_int32, _P]),
    "cutcell_hill_create": (C.c_int, [C.POINTER(CutcellHillDesc), C.POINTER(_P)]),
    "cutcell_hill_skew_conv": (C.c_int, [_P, _P, _P, _P, _P, _P, _P, _P]),
    "cutcell_hill_step": (C.c_int, [_P, _P, _P, _P, _P, C.c_double, C.c_double, _P]),
    "cutcell_hill_destroy": (C.c_int, [_P]),
    "cutcell_batch_create": (C.c_int, [C.c_int32, _P, _P, _P, _P, _P, C.POINTER(_P)]),
    "cutcell_batch_configure": (C.c_int, [_P, C.POINTER(CutcellBatchConfig), _P, _P]),
    "cutcell_batch_info": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "cutcell_batch_solve": (C.c_int, [_P, _P, _P, C.c_double, C.c_int32, C.c_int32, _P, _P]),
    "cutcell_batch_timeline": (C.c_int, [_P, _P, _P, _P]),
    "cutcell_batch_destroy": (C.c_int, [_P]),
    "cutcell_pcg_solve_csr_noalloc": (
        C.c_int,
        [C.c_int32, C.c_int32, _P, _P, _P, _P, _P, C.c_double, C.c_int32, C.c_int32, C.POINTER(CutcellReport), _P],
    ),
    "cutcell_noalloc_last_error": (C.c_char_p, []),
    "cutcell_set_wait_limit": (C.c_int, [C.c_double]),
    "cutcell_kron_create": (C.c_int, [_P, C.POINTER(_P)]),
    "cutcell_apply_form": (C.c_int, [_P, _P, _P, C.c_int32, _P]),
    "cutcell_get_wait_limit": (C.c_double, []),
    "cutcell_barrier_selftest": (C.c_int, [C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "cutcell_status_string": (C.c_char_p, [C.c_int]),
    "cutcell_last_error": (C.c_char_p, []),
}

_lib = None


def load() -> C.CDLL:
    """Load the in-tree shared library (raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("CUTCELL_B200_LIB", LIB_PATH))
    if not path.exists():
        raise CutcellLibraryError(
            f"{path} is missing: build it with `python -m cutcell_b200.build` (nvcc, sm_100a)"
        )
    try:
        lib = C.CDLL(str(path))
    except OSError as exc:  # pragma: no cover - depends on the CUDA runtime
        raise CutcellLibraryError(f"cannot load {path}: {exc}") from exc
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, what: str) -> None:
    if status != OK:
        lib = load()
        msg = lib.cutcell_status_string(status).decode()
        extra = lib.cutcell_last_error().decode()
        raise CutcellLibraryError(f"{what} failed: {msg}" + (f" ({extra})" if extra else ""))


def status_message(status: int) -> str:
    return load().cutcell_status_string(int(status)).decode()


def current_stream_ptr() -> int:
    import torch

    return int(torch.cuda.current_stream().cuda_stream)
