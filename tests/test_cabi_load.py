"""The C-ABI library loads without a GPU and exports every declared symbol."""

import re
from pathlib import Path

from cutcell_b200 import _lib

HEADER = Path(__file__).resolve().parents[1] / "include" / "cutcell_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(cutcell_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_header_symbols():
    lib = _lib.load()
    names = declared_symbols()
    assert names, "no declarations parsed"
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) <= set(_lib.SIGNATURES)


def test_status_strings_match_reference_messages():
    # messages of code/fast_solver_backends.py:245,253-256,263
    assert _lib.status_message(_lib.OK) == "converged"
    assert _lib.status_message(_lib.E_NOCONV) == "maximum iterations reached"
    assert _lib.status_message(_lib.E_BREAKDOWN) == "CG breakdown: non-positive curvature"


def test_solve_spd_has_no_cpu_backend():
    import numpy as np
    import pytest
    import scipy.sparse as sp

    from cutcell_b200 import solve_spd

    with pytest.raises(ValueError):
        solve_spd(sp.eye(3, format="csr"), np.ones(3), backend="cpu")


def test_report_fields_superset_of_reference():
    from dataclasses import fields

    from cutcell_b200 import SolverReport

    names = [f.name for f in fields(SolverReport)]
    ref = ["backend", "method", "preconditioner", "success", "iterations", "elapsed_s", "relative_residual", "message", "transfer_s"]
    assert names[: len(ref)] == ref


def test_wait_limit_setter_validates_and_round_trips():
    lib = _lib.load()
    old = lib.cutcell_get_wait_limit()
    assert 1e-3 <= old <= 3600.0
    assert lib.cutcell_set_wait_limit(0.0) == _lib.E_ARG
    assert lib.cutcell_set_wait_limit(1e9) == _lib.E_ARG
    assert lib.cutcell_set_wait_limit(2.5) == _lib.OK
    assert abs(lib.cutcell_get_wait_limit() - 2.5) < 1e-9
    assert lib.cutcell_set_wait_limit(old) == _lib.OK
