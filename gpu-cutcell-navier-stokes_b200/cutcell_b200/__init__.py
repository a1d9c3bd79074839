"""cutcell_b200: B200 (sm_100a) solve path for aggregated cut-cell B-spline systems.

Host side: geometry / element setup (``problem``, ``cutgeom``, ``bspline``),
aggregation ``E`` (``aggregation``), the tile layout and device operator
(``operator``) and the reference-compatible solver entry points
(``fast_solver_backends.solve_spd``).  Device side: libcutcell_b200.so,
loaded through ``_lib`` (C ABI in include/cutcell_b200.h).
"""

from .fast_solver_backends import SolverReport, as_csr, csr_memory_bytes, make_linear_solver, solve_spd  # noqa: F401

__all__ = ["SolverReport", "as_csr", "csr_memory_bytes", "make_linear_solver", "solve_spd"]
