"""CPU oracle for the cut-cell solve path -- TEST INFRASTRUCTURE ONLY.

This package restates, on the CPU, the reference algorithms that the B200
library replaces, each function citing the reference file:line it follows.
It is the checker: only ``tests/``, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of ``bench.py`` may import it.
The product package never imports it and has no CPU solver of its own.

Pinning: the restatements are checked against golden vectors produced by the
reference's own Python code (``tests/golden/make_golden.py``) and against the
reference's committed result files (iteration counts and unknown counts in
benchmarks/results/gpu_solver_benchmark_3d.csv and
code/results/fast_solver_stress.csv).
"""
