"""Benchmark: seconds per PCG solve to relative residual 1e-9 on the
sphere-cut Poisson problem (p = 3, 32 elements per axis, r = 0.31), B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one complete solve of the aggregated system E^T A E x = E^T f from
x = 0 to ||r||/||b|| <= 1e-9, inputs resident in HBM.  The L2 cache (126 MB) is
flushed between timed solves by writing a 256 MB buffer.  Variants measured:
plain FP64 Jacobi-PCG (the default form), FP64 iterative refinement around
FP32 / BF16 operator applies, and flexible PCG with the learned patch
correction (trained in this run on random radii in [0.2, 0.4] by the
project's kernels); ``value`` is the fastest variant that reaches the
tolerance, every variant is listed under ``variants``.  Multi-GPU: independent
replicas (one solve per rank per step, no collective on the data path).

``--impl reference`` times the reference's CPU path (SciPy Jacobi-CG on the
assembled CSR E^T A E, restated in oracle/pcg.py) on the host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "gpu-cutcell-navier-stokes_b200"))
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "s per PCG solve to rel. residual 1e-9: learned/mixed vs FP64 Jacobi, 1 B200"
UNIT = "s/solve"
TOL = 1e-9


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--p", type=int, default=3)
    ap.add_argument("--radius", type=float, default=0.31)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variants", default="fp64,fp32-ir,bf16-ir,block,learned,twolevel")
    ap.add_argument("--no-extras", action="store_true", help="skip the batch / hill-step / cut-box summaries of the default run")
    ap.add_argument("--train-geometries", type=int, default=3)
    ap.add_argument("--train-pairs", type=int, default=20000)
    ap.add_argument("--workload", default="sphere", choices=["sphere", "hill", "hill-step", "batch", "apply", "cut-box"])
    ap.add_argument("--cutbox-n", type=int, default=64)
    ap.add_argument("--batch-count", type=int, default=72)
    ap.add_argument("--hill-nr", type=int, default=2345)
    ap.add_argument("--hill-nz", type=int, default=32)
    ap.add_argument("--hill-nex", type=int, default=64)
    ap.add_argument("--hill-ney", type=int, default=32)
    ap.add_argument("--hill-build", default="real", choices=["real", "synthetic"])
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    Q = (
        "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
        "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
        "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"
    )

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(
                    ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits"],
                    capture_output=True, text=True, timeout=5,
                ).stdout.strip()
                if out:
                    self.rows.append([c.strip() for c in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def start(self):
        """Starts sampling a timed region; a sampler may cover several regions in turn."""
        self._stop.clear()
        self._mark = len(self.rows)
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def stop(self):
        """Ends the current region and returns the record of its samples."""
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
            self._t = None
        return self.summary(self.rows[getattr(self, "_mark", 0):])

    def total(self):
        """The record of every region this sampler covered."""
        return self.summary(self.rows)

    @staticmethod
    def summary(rows):
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i] and "Not" not in r[5 + i]})
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(mx)) if mx else None,
            "reasons": reasons,
            "samples": len(rows),
        }


# DRAM bytes (read + write) per launch of each workload's dominant kernel, from
# one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of the same
# command; None where no capture was made for that configuration.
NCU_TRAFFIC = {
    ("sphere", 32, 3): 37.10e6 + 1.50e6,   # pcg_kernel, one whole solve
    ("sphere-twolevel", 32, 3): 410.43e6 + 42.31e6,  # tlpcg_kernel (four patch tilings, BF16 inverses), one whole solve
    ("sphere-block", 32, 3): 131.61e6 + 7.13e6,      # ppcg_kernel (exact patch blocks), one whole solve
    ("cut-box", 64, 3): 2.38e6,                      # apply_kernel<KronOp>, one apply
    ("apply", 64, 3): 157.17e6 + 6.61e6,   # apply_kernel, one apply
    ("batch", 72): 17.6e6,                 # batch_pcg_kernel, one launch
    ("hill-step",): 245.29e6 + 55.68e6,    # hill_segment_kernel, one 3-component advection (64x32x32 channel, single launch)
}


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def host_cpu() -> dict:
    """The host the CPU baseline ran on: logical CPUs and the CPU model name."""
    model = "unknown"
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return {"nproc": os.cpu_count() or 1, "cpu_model": model}


def cut_block_entries(P: int) -> int:
    """Stored entries per cut-element block: degree 3 (P = 64) keeps the upper
    triangle of its symmetric block (P(P+1)/2), other degrees the dense block."""
    return P * (P + 1) // 2 if P == 64 else P * P


def algorithmic_bytes_per_iter(prob, ext, prec: str) -> float:
    """B_iter = 13*8*N_red + B_E + B_op (FP64 vectors, E gather + scatter,
    stored per-cut-element blocks in the operator's storage precision)."""
    N = ext.n_red
    nnz_small = int(ext.E[ext.small_support].nnz)
    b_e = 2 * (4 + 8) * nnz_small + 4 * ext.n_full
    s = {"fp64": 8, "fp32-ir": 4, "bf16-ir": 4}[prec]  # bf16-ir: two BF16 planes per entry
    b_op = prob.cut_ids.size * cut_block_entries(prob.P) * s
    return 13 * 8 * N + b_e + b_op


def algorithmic_bytes_patch(prob, ext, n_patch: int, ncg: int = 0, extra_patches=()) -> float:
    """Per iteration of the patch-preconditioned solves: the FP64 operator
    streams of one apply (B_E + B_op) once (exact blocks) or twice (two-level:
    A p and A zc), the patch inverses (4096 entries per patch: FP64 for the
    exact-block form, BF16 for the two-level form, which also reads the
    extra tilings'), the dense coarse inverse (FP64, 8 ncg^2), and the FP64
    vector streams (13 N for one apply's PCG; the two-level form adds the
    line update, prolongation, second apply and the patch step: 20 N, and
    6 N more per extra tiling: its z written and read twice, r, A zc and
    r_old read again)."""
    N = ext.n_red
    nnz_small = int(ext.E[ext.small_support].nnz)
    b_e = 2 * (4 + 8) * nnz_small + 4 * ext.n_full
    b_op = prob.cut_ids.size * cut_block_entries(prob.P) * 8
    if ncg:
        # the second tiling adds its inverses, z2 written and read, and r, A zc, r_old read again
        # the two-level form stores its patch inverses in BF16, Ac^-1 in FP64
        nx = len(extra_patches)
        return (2 * (b_e + b_op) + (20 + 6 * nx) * 8 * N + 2 * 4096 * (n_patch + sum(extra_patches))
                + 8 * ncg * ncg)
    return (b_e + b_op) + 13 * 8 * N + 8 * 4096 * n_patch


def cpu_baseline(prob, ext, b, sample_solves=1):
    """Reference CPU path (SciPy Jacobi-CG, 1 thread) on the assembled CSR."""
    from oracle.aggregation import restrict_spd
    from oracle.pcg import solve_cpu_cg

    A = restrict_spd(prob.assemble_full_csr(), ext.E)
    times, its = [], []
    for _ in range(sample_solves):
        t0 = time.perf_counter()
        x, rep = solve_cpu_cg(A, b, tol=TOL, maxiter=20000)
        times.append(time.perf_counter() - t0)
        its.append(rep["iterations"])
    return A, float(np.mean(times)), int(its[0]), x


BATCH_METRIC = "solves/s: uneven oblique-cut Jacobi-PCG systems solved to rel. residual 1e-9 in one persistent launch"


def batch_systems(count: int):
    """The batched workload: ``count`` 2D oblique cuts (angle U[0,45] deg,
    offset U(0,h), p in {3,4,5}, n in {6,8,12,16,24}, mass or stiffness),
    N(0,1) right-hand sides; seeded."""
    from cutcell_b200 import oblique2d as ob

    cases = ob.sample_cases(count, seed=20260629)
    systems = [ob.build_oblique(*c).A for c in cases]
    rng = np.random.default_rng(12345)
    rhs = [rng.standard_normal(A.shape[0]) for A in systems]
    return cases, systems, rhs


def run_batch_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle.pcg import solve_cpu_cg

    _, systems, rhs = batch_systems(args.batch_count)
    for _ in range(min(args.warmup, 1)):
        for A, b in zip(systems, rhs):
            solve_cpu_cg(A, b, tol=TOL, maxiter=20000)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        for A, b in zip(systems, rhs):
            solve_cpu_cg(A, b, tol=TOL, maxiter=20000)
        ts.append(time.perf_counter() - t0)
    v = len(systems) / float(np.mean(ts))
    line = {
        "impl": "reference", "metric": BATCH_METRIC, "value": v, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(ts)) * 1e3, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cuts and right-hand sides)",
        "config": {"workload": f"{len(systems)} oblique 2D cut systems, one solve_cpu_cg each"},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": 1, "kind": "port",
                         "sample": f"all {len(systems)} systems per step, sequential SciPy CG", **host_cpu()},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args, rank, world, local, emit=True):
    """72 uneven systems in one persistent, graph-captured launch (per rank:
    its longest-processing-time share when several GPUs are used).  With
    emit=False the JSON line is returned instead of printed."""
    import torch

    from cutcell_b200.batch import BatchSolver, partition_lpt
    from cutcell_b200.fast_solver_backends import CsrDeviceMatrix

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1 and emit:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    t_setup = time.perf_counter()
    cases, systems, rhs = batch_systems(args.batch_count)
    t_setup = time.perf_counter() - t_setup
    costs = [A.nnz * np.sqrt(A.shape[0]) for A in systems]
    mine = partition_lpt(costs, world)[rank]
    sys_m = [systems[i] for i in mine]
    rhs_m = [rhs[i] for i in mine]
    bs = BatchSolver(sys_m, device=dev)
    bs.rhs.copy_(torch.from_numpy(bs.packed.pack(rhs_m)))
    t0 = time.perf_counter()
    best = bs.autotune(tol=TOL, maxiter=20000)
    tune_s = time.perf_counter() - t0
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        reps = bs.solve_device(tol=TOL, maxiter=20000)
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        barrier()
        reps = bs.solve_device(tol=TOL, maxiter=20000)  # device time of the captured graph (CUDA events)
        ms.append(float(reps[0].elapsed_ms))
    barrier()
    clocks = sampler.stop()
    tot = float(np.sum(ms))
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([tot], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot = float(t.item())
    ms_step = tot / args.steps
    value = len(systems) / (ms_step / 1e3)
    its = np.array([r.iterations for r in reps])
    ok = all(r.status == 0 and r.true_relative_residual <= 10 * TOL for r in reps)
    tl = bs.timeline()
    dur = tl["end_us"] - tl["start_us"]
    pk = bs.packed
    bytes_alg = float(np.sum(its * (12.0 * pk.nnz + 13.0 * 8.0 * pk.n)))
    hbm, hbm_kind = peaks()
    achieved = bytes_alg / (ms_step / 1e3) / 1e9

    # 72 sequential plain solves through the single-system device path
    seq_ms, seq_its = 0.0, 0
    for A, b in zip(sys_m, rhs_m):
        M = CsrDeviceMatrix(A, device=dev)
        bd = torch.as_tensor(b).to(dev)
        M.solve_device(bd, tol=TOL, maxiter=20000)
        _, r = M.solve_device(bd, tol=TOL, maxiter=20000)
        seq_ms += float(r.elapsed_ms)
        seq_its += int(r.iterations)
        M.close()

    # end to end through the public API: host vectors in (pinned staging, H2D),
    # host solutions out (D2H), per step
    for _ in range(2):
        bs.solve(rhs_m, tol=TOL, maxiter=20000)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        out = bs.solve(rhs_m, tol=TOL, maxiter=20000)
    barrier()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    nvec = int(pk.vec_off[-1])
    line = {
        "metric": BATCH_METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "strong" if world > 1 else "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded cuts and N(0,1) right-hand sides)",
        "config": {
            "workload": f"{len(systems)} oblique 2D cut systems (p 3-5, n 6-24, mass/stiffness), Jacobi-PCG to {TOL}",
            "n_total": int(sum(A.shape[0] for A in systems)), "nnz_total": int(sum(A.nnz for A in systems)),
            "systems_this_rank": len(sys_m), "autotuned": str(best), "teams": bs.info()["teams"], "tune_s": tune_s,
            "iterations_total": int(its.sum()), "iterations_max": int(its.max()),
            "critical_system_us": float(dur.max()), "all_converged": bool(ok), "setup_s": t_setup,
            "l2": "flushed between timed launches (256 MB write)", "parallelism": f"LPT partition x{world}",
        },
        "sequential": {"ms": seq_ms, "solves_per_s": len(sys_m) / (seq_ms / 1e3), "iterations": seq_its,
                       "path": "one cutcell_pcg_solve (CSR, persistent cooperative launch) per system"},
        "clocks": clocks,
        "e2e": {"value": len(systems) / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": 8 * nvec,
                "d2h_bytes_per_step": 8 * nvec},
        "gpu_launches": int(args.steps),
        "roofline": {"bound": "hbm", "kernel": "batch_pcg_kernel (whole batch, one launch)", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": hbm_kind,
                     "traffic": NCU_TRAFFIC.get(("batch", args.batch_count)), "algorithmic_bytes": bytes_alg,
                     "note": "algorithmic bytes per iteration 12 nnz + 13*8 n; the CSR slices and vectors are held in shared memory"},
    }
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        from oracle.pcg import solve_cpu_cg

        t0 = time.perf_counter()
        k = 0
        while k < len(systems) and time.perf_counter() - t0 < 20.0:
            solve_cpu_cg(systems[k], rhs[k], tol=TOL, maxiter=20000)
            k += 1
        cs = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": k / cs, "unit": "solves/s", "cores": 1, "kind": "port",
                                "sample": f"first {k} of the {len(systems)} systems, sequential SciPy CG", **host_cpu()}
    if not emit:
        bs.close()
        return line
    if rank == 0:
        print(json.dumps(line), flush=True)
    bs.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_reference(args, rank, world):
    if args.workload == "batch":
        return run_batch_reference(args, rank, world)
    if rank != 0:
        return 0
    nth = os.cpu_count() or 1
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = str(nth)
    from cutcell_b200.workloads import sphere_poisson
    from oracle.aggregation import restrict_spd
    from oracle.pcg import solve_cpu_cg

    # the system is built by the NumPy host setup (no native library of this
    # package is loaded in this arm) and assembled by the oracle
    from oracle.assembly import assemble_full

    t_setup = time.perf_counter()
    prob, ext = sphere_poisson(args.n, args.p, args.radius, native=False)
    b = np.asarray(ext.E.T @ prob.load)
    A = restrict_spd(assemble_full(prob), ext.E)
    t_setup = time.perf_counter() - t_setup
    for _ in range(args.warmup):
        solve_cpu_cg(A, b, tol=TOL, maxiter=20000)
    ts = []
    it = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, rep = solve_cpu_cg(A, b, tol=TOL, maxiter=20000)
        ts.append(time.perf_counter() - t0)
        it = rep["iterations"]
    v = float(np.mean(ts))
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": v,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": v * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded geometry, manufactured forcing)",
        "config": {"workload": f"sphere-cut Poisson p={args.p} n={args.n} r={args.radius}", "n_red": ext.n_red, "nnz": int(A.nnz), "iterations": it,
                   "setup": "NumPy cut quadrature + oracle assembly (no native code of this package)", "setup_s": t_setup},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port", "sample": "full solve per step (SciPy CSR SpMV is single-threaded)", **host_cpu()},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_hill(args, rank, world, local):
    """Fast-diagonalisation solve at the hill configuration's sizes: nr reduced
    2D modes (2345 for 64x32 elements, p=3), nz = 32 spanwise modes.  The
    operators are seeded synthetic matrices of those shapes (the reference's
    hill builder is isotropic and builds the inverses in hours on the CPU);
    the timed work is the full FastDiagHill::solve data flow."""
    import torch

    from cutcell_b200.hill import FastDiagHill

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nr, nz = args.hill_nr, args.hill_nz
    g = torch.Generator(device=dev).manual_seed(20260629)
    rnd = lambda *shape: torch.randn(*shape, generator=g, device=dev, dtype=torch.float64) / np.sqrt(shape[-1])
    M2, Qx2, Qy2 = rnd(nr, nr), rnd(nr, nr), rnd(nr, nr)
    kz = np.arange(nz)
    Mz_row = np.zeros(nz); Mz_row[0], Mz_row[1], Mz_row[-1] = 0.6, 0.2, 0.2
    Sz_row = np.zeros(nz); Sz_row[0], Sz_row[1], Sz_row[-1] = 2.0, -1.0, -1.0
    Kz_row = np.zeros(nz); Kz_row[1], Kz_row[-1] = 0.5, -0.5
    Ainv, Sinv = rnd(nz, nr, nr), rnd(nz, nr, nr)
    fd = FastDiagHill(device=dev).build(M2, Qx2, Qy2, None, Mz_row, Sz_row, Kz_row, 0.01, inverses=(Ainv, Sinv))
    u = [rnd(nr, nz) for _ in range(3)]
    out = [torch.empty_like(u[0]) for _ in range(3)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        fd.solve_device(*u, out=out)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ms = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fd.solve_device(*u, out=out)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    t = float(np.mean(ms))
    bytes_inv = 3 * nz * nr * nr * 8
    hbm, kind = peaks()
    achieved = bytes_inv / (t / 1e3) / 1e9
    line = {
        "metric": "ms per hill fast-diagonalisation solve (FastDiagHill::solve data flow)",
        "value": t, "unit": "ms/solve", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic operators of the configuration's sizes (seeded)",
        "config": {"workload": f"hill fast-diag nr={nr} nz={nz}", "l2": "flushed between timed solves"},
        "clocks": clocks, "gpu_launches": 15 * args.steps,
        "roofline": {"bound": "hbm", "kernel": "fd_mode_mv_kernel (Ainv twice, Sinv once)", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": kind, "traffic": None,
                     "algorithmic_bytes": bytes_inv},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    fd.close()
    return 0


def run_hill_step(args, rank, world, local, emit=True):
    """One hill_fastdiag_step (SSP-RK3 skew advection + fast-diagonalisation
    solve) on the periodic-hill channel: 64 x 32 x-y elements, nz = 32,
    p = 3, physical metric (Lx = 9, Ly = 3.036, Lz = 4.5), nu = 1/5600,
    dt = 0.02, from the parabolic initial condition with a 1 % perturbation.
    The channel is built by the anisotropic restatement of Hill3D::build
    (cutcell_b200.hillsetup) and its per-mode operators on the device through
    the shared eigenbasis.  ``--hill-build synthetic`` times seeded stand-ins
    of the same shapes instead."""
    import torch

    from cutcell_b200.hill import FastDiagHill, HillAdvection, synthetic_machinery

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    nz = args.hill_nz
    t0 = time.perf_counter()
    dt, nu = 0.02, 1.0 / 5600.0
    hs = None
    if args.hill_build == "real":
        from cutcell_b200.hillsetup import build_hill, parabolic_ic

        hs = build_hill(args.hill_nex, args.hill_ney, 3, nz, 4.5, physical=True)
        host_build_s = time.perf_counter() - t0
        m = hs.machinery()
        nr = hs.nr
        adv = HillAdvection(m["phi"], m["dpx"], m["dpy"], m["w2"], m["Vz"], m["dVz"], m["wz"], m["M2inv"],
                            m["Mzinv"], device=dev)
        fd = FastDiagHill(device=dev).build(hs.M2, hs.Qx2, hs.Qy2, hs.KN2, hs.Mz[0], hs.Sz[0], hs.Kz[0], dt * nu,
                                            on_device=True)
        u0 = [torch.as_tensor(np.ascontiguousarray(c)).to(dev) for c in parabolic_ic(hs)]
        setup_s = time.perf_counter() - t0
    else:
        nr = args.hill_nr
        m = synthetic_machinery(nr=nr, nz=nz, cells=(64, 32), pts_per_cell=196, modes_per_row=16)
        adv = HillAdvection(m["phi"], m["dpx"], m["dpy"], m["w2"], m["Vz"], m["dVz"], m["wz"], m["M2inv"],
                            m["Mzinv"], device=dev)
        g = torch.Generator(device=dev).manual_seed(20260629)
        rnd = lambda *shape: torch.randn(*shape, generator=g, device=dev, dtype=torch.float64) / np.sqrt(shape[-1])
        M2, Qx2, Qy2 = rnd(nr, nr), rnd(nr, nr), rnd(nr, nr)
        Mz_row = np.zeros(nz); Mz_row[0], Mz_row[1], Mz_row[-1] = 0.6, 0.2, 0.2
        Sz_row = np.zeros(nz); Sz_row[0], Sz_row[1], Sz_row[-1] = 2.0, -1.0, -1.0
        Kz_row = np.zeros(nz); Kz_row[1], Kz_row[-1] = 0.5, -0.5
        Ainv, Sinv = rnd(nz, nr, nr), rnd(nz, nr, nr)
        fd = FastDiagHill(device=dev).build(M2, Qx2, Qy2, None, Mz_row, Sz_row, Kz_row, 0.01, inverses=(Ainv, Sinv))
        u0 = [0.1 * rnd(nr, nz) for _ in range(3)]
        host_build_s = 0.0
        setup_s = time.perf_counter() - t0
    u = [t.clone() for t in u0]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        for a, b in zip(u, u0):
            a.copy_(b)
        adv.step(fd, u, dt, 0.0)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    ms, ms_adv = [], []
    for _ in range(args.steps):
        for a, b in zip(u, u0):
            a.copy_(b)
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        adv.step(fd, u, dt, 0.0)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
        flush.fill_(1.0)
        torch.cuda.synchronize()
        e0.record()
        adv.skew_conv(*u0)
        e1.record()
        torch.cuda.synchronize()
        ms_adv.append(e0.elapsed_time(e1))
    clocks = sampler.stop()
    t = float(np.mean(ms))
    ta = float(np.mean(ms_adv))
    n2q, nzq = m["phi"].shape[0], m["Vz"].shape[0]
    L = round(m["phi"].nnz / n2q)
    # FP64 flops of one skew_conv of three components (fused kernel), per 2D point:
    # 2D sample 9 L nz FMA, z band 3 x (qpe x nz) x (48 + 12 FMA + ~10), 2D load 9 L nz FMA
    flop_adv = 2.0 * n2q * (18 * L * nz + 3 * nzq * 70) + 2.0 * nr * nr * 3 * nz
    div = None
    if hs is not None:
        from cutcell_b200.hillsetup import weak_div

        uh = [c.cpu().numpy() for c in u]
        d0 = float(np.abs(weak_div(hs, *[c.cpu().numpy() for c in u0])).max())
        d1 = float(np.abs(weak_div(hs, *uh)).max())
        div = {"max_abs_initial": d0, "max_abs_after_step": d1, "ratio": d1 / d0,
               "max_abs_u": float(max(np.abs(c).max() for c in uh)),
               "note": "weak divergence hill_weak_div (hill3d.h:330-334) of the stepped velocity"}
    line = {
        "metric": "ms per hill fast step (SSP-RK3 skew advection + fast-diagonalisation solve)",
        "value": t, "unit": "ms/step", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": ("periodic-hill channel built by the anisotropic Hill3D::build restatement, parabolic IC + 1 % seeded "
                 "perturbation" if hs is not None else "synthetic sample machinery and operators of the configuration's sizes (seeded)"),
        "config": {"workload": (f"hill channel {args.hill_nex}x{args.hill_ney} elements nz={nz} p=3 physical metric "
                                f"(nr={nr} n2q={n2q} nzq={nzq} row_nnz={L})" if hs is not None else
                                f"hill fast step nr={nr} nz={nz} n2q={n2q} nzq={nzq} row_nnz={L}"),
                   "l2": "flushed between timed steps", "setup_s": setup_s, "host_build_s": host_build_s,
                   "fastdiag_build": getattr(fd, "build_timings", None), "advect_ms": ta,
                   "advect_gflops": flop_adv / (ta * 1e-3) / 1e9, "divergence": div, "dt": dt, "nu": nu},
        "clocks": clocks, "gpu_launches": (3 * 4 + 3 + 15) * args.steps,
        # the advection kernel is FP64-FMA bound (no tensor-core FP64 kind on this path);
        # peak: B200 FP64 nominal, not measured on this pool
        "roofline": {"bound": "fp64", "kernel": "hill_segment_kernel (one 3-component advection)",
                     "achieved": flop_adv / (ta * 1e-3) / 1e12, "peak": 37.0, "unit": "TFLOP/s",
                     "frac": flop_adv / (ta * 1e-3) / 1e12 / 37.0, "peak_kind": "nominal",
                     "traffic": NCU_TRAFFIC.get(("hill-step",))},
    }
    if not emit:
        adv.close()
        fd.close()
        return line
    if rank == 0:
        print(json.dumps(line), flush=True)
    adv.close()
    fd.close()
    return 0


def run_apply(args, rank, world, local):
    """The matrix-free operator apply y = E^T A E x alone (one cooperative
    launch per apply), FP64 / FP32 / BF16 operator storage, L2 flushed
    between applies.  Algorithmic bytes per apply: x in and y out (FP64),
    the E small rows and index maps, and the stored cut-element blocks."""
    import torch

    from cutcell_b200.operator import CutCellOperator
    from cutcell_b200.workloads import sphere_poisson

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    t0 = time.perf_counter()
    prob, ext = sphere_poisson(args.n, args.p, args.radius)
    op = CutCellOperator(prob, ext, device=dev)
    setup_s = time.perf_counter() - t0
    g = torch.Generator(device=dev).manual_seed(7)
    x = torch.randn(ext.n_red, generator=g, device=dev, dtype=torch.float64)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    hbm, kind = peaks()
    nnz_small = int(ext.E[ext.small_support].nnz)
    P = (args.p + 1) ** 3
    out = {}
    for prec, s in (("fp64", 8), ("fp32-ir", 4), ("bf16-ir", 2)):
        for _ in range(args.warmup):
            op.apply(x, precision=prec)
        torch.cuda.synchronize()
        ms = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            op.apply(x, precision=prec)
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        t = float(np.median(ms))
        nbytes = 2 * 8 * ext.n_red + 2 * (4 + 8) * nnz_small + 4 * ext.n_full + prob.cut_ids.size * cut_block_entries(P) * s
        out[prec] = {"ms": t, "bytes": nbytes, "GBps": nbytes / (t / 1e3) / 1e9, "frac": nbytes / (t / 1e3) / 1e9 / hbm}
    line = {
        "metric": "operator apply y = E^T A E x (matrix-free), GB/s of algorithmic bytes",
        "value": out["fp64"]["GBps"], "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": out["fp64"]["ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded geometry)",
        "config": {"workload": f"sphere-cut apply p={args.p} n={args.n}", "n_red": ext.n_red, "n_cut_elements": int(prob.cut_ids.size),
                   "setup_s": setup_s, "l2": "flushed between applies"},
        "variants": out,
        "roofline": {"bound": "hbm", "kernel": "apply_kernel<TileOp<double>>", "achieved": out["fp64"]["GBps"], "peak": hbm,
                     "unit": "GB/s", "frac": out["fp64"]["frac"], "peak_kind": kind,
                     "traffic": NCU_TRAFFIC.get(("apply", args.n, args.p)), "algorithmic_bytes": out["fp64"]["bytes"]},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    op.close()
    return 0


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "hill":
        return run_hill(args, rank, world, local)
    if args.workload == "batch":
        return run_batch(args, rank, world, local)
    if args.workload == "hill-step":
        return run_hill_step(args, rank, world, local)
    if args.workload == "apply":
        return run_apply(args, rank, world, local)
    if args.workload == "cut-box":
        return run_cutbox_line(args, rank, world, local)
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from cutcell_b200 import solve_spd
    from cutcell_b200.operator import CutCellOperator
    from cutcell_b200.workloads import sphere_poisson

    t_setup = time.perf_counter()
    prob, ext = sphere_poisson(args.n, args.p, args.radius)
    op = CutCellOperator(prob, ext, device=dev)
    t_setup = time.perf_counter() - t_setup
    b_host = np.asarray(ext.E.T @ prob.load)
    b = torch.as_tensor(b_host).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize(dev)

    variants = {}
    ref_x = None
    learned_info = None
    wanted = args.variants.split(",")
    if "learned" in wanted:
        # training on random sphere radii in [0.2, 0.4] with the project's kernels
        from cutcell_b200.learned import PatchMLP, attach, attach_blocks, fit_linear, generate_pairs, train

        t0 = time.perf_counter()
        rng = np.random.default_rng(20260629)
        radii = [float(r) for r in rng.uniform(0.2, 0.4, args.train_geometries)]
        train_ops = [CutCellOperator(*sphere_poisson(args.n, args.p, r), device=dev) for r in radii]
        X, T = generate_pairs(train_ops, args.train_pairs, seed=11)
        # least-squares start of the identity-activation network, then Adam
        # fine-tuning with the project's training kernels
        net = PatchMLP(fit_linear(X, T), activation="identity")
        hist = train(net, X, T, epochs=4, batch=512, lr=1e-5)
        attach(op, net)
        for o in train_ops:
            o.close()
        learned_info = {"radii": radii, "pairs": int(X.shape[0]), "loss_first": hist[0], "loss_last": hist[-1],
                        "target_mean_square": float((T.double() ** 2).mean()), "train_s": time.perf_counter() - t0,
                        "canonical_patches": int(op._patch_solves.canonical.sum()) if hasattr(op, "_patch_solves") else None}
    t_blocks = None
    t_coarse = None
    # one sampler over every variant's timed region (and only those): each
    # variant keeps its own record, the line's record is the union
    sampler = ClockSampler(local)
    for prec in wanted:
        solve_kw = {"precision": prec}
        if prec == "twolevel":
            from cutcell_b200.coarse import attach_coarse
            from cutcell_b200.learned import attach_blocks

            attach_blocks(op, "all")
            t0 = time.perf_counter()
            cl = attach_coarse(op)
            t_coarse = {"setup_s": time.perf_counter() - t0, "galerkin_s": cl.galerkin_s, "factor": cl.factor,
                        "coarse_dofs": int(cl.keep.size), "minv_bytes": int(8 * cl.ncg * cl.ncg),
                        "extra_tilings": {"shifts": list(cl.shifts), "patches": [int(t.n_patch) for t in cl.extra]},
                        "omega": cl.omega}
            solve_kw = {"precision": "fp64", "preconditioner": "twolevel"}
        elif prec in ("learned", "block"):
            from cutcell_b200.learned import attach_blocks

            t0 = time.perf_counter()
            attach_blocks(op, "noncanonical" if prec == "learned" else "all")
            t_blocks = t_blocks or time.perf_counter() - t0
            solve_kw = {"precision": "fp64", "preconditioner": "jacobi+learned" if prec == "learned" else "block"}
        elif prec != "fp64":
            op.set_refinement(0.1)
        for _ in range(args.warmup):
            x, rep = op.solve_device(b, tol=TOL, maxiter=20000, **solve_kw)
        barrier()
        sampler.start()
        ms = []
        for _ in range(args.steps):
            flush.fill_(1.0)
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            x, rep = op.solve_device(b, tol=TOL, maxiter=20000, **solve_kw)
            e1.record()
            torch.cuda.synchronize(dev)
            ms.append(e0.elapsed_time(e1))
        barrier()
        clocks = sampler.stop()
        tot = float(np.sum(ms))
        if world > 1:
            import torch.distributed as dist

            t = torch.tensor([tot], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            tot = float(t.item())
        xs = x.double().cpu().numpy()
        if prec == "fp64":
            ref_x = xs
        variants[prec] = {
            "s_per_solve": tot / 1e3 / args.steps,
            "iterations": int(rep.iterations),
            "outer_iterations": int(rep.outer_iterations),
            "true_relative_residual": float(rep.true_relative_residual),
            "converged": bool(rep.status == 0 and rep.true_relative_residual <= TOL * 10),
            "rel_err_vs_fp64": float(np.linalg.norm(xs - ref_x) / np.linalg.norm(ref_x)) if ref_x is not None else None,
            "kernel_ms": float(np.mean(ms)),
            "blocks": int(rep.blocks),
        }
        if clocks:
            variants[prec]["clocks"] = clocks
        if prec == "learned" and learned_info:
            variants[prec]["training"] = learned_info
    plain = variants["fp64"]
    ok = {k: v for k, v in variants.items() if v["converged"]}
    best_key = min(ok, key=lambda k: ok[k]["s_per_solve"]) if ok else "fp64"
    best = variants[best_key]

    # end-to-end through the public API, host buffers (pinned), H2D + D2H inside
    b_pin = torch.from_numpy(b_host).pin_memory()
    e2e_prec = best_key
    e2e_kw = {"precision": e2e_prec}
    if e2e_prec == "learned":
        e2e_kw = {"preconditioner": "jacobi+learned"}
    elif e2e_prec == "block":
        e2e_kw = {"preconditioner": "block"}
    elif e2e_prec == "twolevel":
        e2e_kw = {"preconditioner": "twolevel"}
    for _ in range(2):
        solve_spd(op, b_pin.numpy(), tol=TOL, maxiter=20000, **e2e_kw)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        x_host, rep_h = solve_spd(op, b_pin.numpy(), tol=TOL, maxiter=20000, **e2e_kw)
    torch.cuda.synchronize(dev)
    e2e = (time.perf_counter() - t0) / args.steps

    hbm, hbm_kind = peaks()
    bytes_iter = algorithmic_bytes_per_iter(prob, ext, "fp64")
    achieved = bytes_iter * plain["iterations"] / (plain["kernel_ms"] / 1e3) / 1e9
    roof_plain = {"bound": "hbm", "kernel": "pcg_kernel<TileOp<double>> (plain FP64, whole solve)",
                  "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": hbm_kind,
                  "traffic": NCU_TRAFFIC.get(("sphere", args.n, args.p)), "traffic_per": "launch (one solve)",
                  "bytes_per_iter": bytes_iter}
    # the roofline of the headline variant's kernel
    roof = roof_plain
    if best_key in ("twolevel", "block") and hasattr(op, "_patches"):
        npatch = int(op._patches.n_patch)
        ncg = int(op._coarse.ncg) if best_key == "twolevel" else 0
        extra = [int(t.n_patch) for t in op._coarse.extra] if best_key == "twolevel" else []
        b_it = algorithmic_bytes_patch(prob, ext, npatch, ncg, extra)
        ach = b_it * best["iterations"] / (best["kernel_ms"] / 1e3) / 1e9
        roof = {"bound": "hbm",
                "kernel": ("tlpcg_kernel<TileOp<double,4>> (two-level flexible PCG, whole solve)" if best_key == "twolevel"
                           else "ppcg_kernel<TileOp<double,4>> (exact patch blocks, whole solve)"),
                "achieved": ach, "peak": hbm, "unit": "GB/s", "frac": ach / hbm, "peak_kind": hbm_kind,
                "traffic": NCU_TRAFFIC.get(("sphere-" + best_key, args.n, args.p)), "traffic_per": "launch (one solve)",
                "bytes_per_iter": b_it,
                "note": "algorithmic bytes mostly served from L2 (traffic = ncu DRAM bytes of one launch)"}
    line = {
        "metric": METRIC,
        "value": best["s_per_solve"],
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": best["s_per_solve"] * 1e3,
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded geometry, manufactured forcing)",
        "config": {
            "workload": f"sphere-cut Poisson p={args.p} n={args.n} r={args.radius} (matrix-free E^T A E)",
            "n_red": ext.n_red,
            "n_full": ext.n_full,
            "n_cut_elements": int(prob.cut_ids.size),
            "min_cut_fraction": prob.min_cut_fraction,
            "tol": TOL,
            "headline_variant": best_key,
            "l2": "flushed between timed solves (256 MB write)",
            "parallelism": f"replicas x{world}",
            "setup_s": t_setup,
        },
        "variants": variants,
        "clocks": dict(sampler.total(), regions="the timed solves of every variant"),
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(8 * ext.n_red), "d2h_bytes_per_step": int(8 * ext.n_red), "variant": e2e_prec},
        "gpu_launches": int(args.steps),
        "roofline": roof,
        "roofline_plain_fp64": roof_plain,
    }
    if rank == 0 and not args.no_cpu_baseline and world == 1:
        A, cpu_s, cpu_it, xc = cpu_baseline(prob, ext, b_host)
        line["cpu_baseline"] = {
            "value": cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"one full SciPy Jacobi-CG solve on the assembled CSR (nnz {A.nnz}, {cpu_it} iterations)",
            **host_cpu(),
        }
        line["config"]["cpu_rel_err_vs_gpu_fp64"] = float(np.linalg.norm(xc - ref_x) / np.linalg.norm(xc))
    if t_blocks is not None:
        line["config"]["patch_blocks_setup_s"] = t_blocks
    if t_coarse is not None:
        line["config"]["coarse_level"] = t_coarse
    if world == 1 and not args.no_extras:
        line["extras"] = extras_summary(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    op.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_cutbox(args, dev, steps: int, n: int = 64, p: int = 3, warmup: int = 3):
    """The tensor cut-box Poisson system of solve_poisson_3d (cuts at
    fractions 0.6 on all three axes) solved matrix-free with the Kronecker
    operator: Jacobi-PCG to 1e-9 (device time) and one apply of the Poisson
    form, L2 flushed between launches."""
    import torch

    from cutcell_b200 import tensorbox as tb

    t0 = time.perf_counter()
    box = tb.cut_box(n, p, (0.6, 0.6, 0.6))
    rhs = tb.poisson_rhs(box)
    op = tb.KronOperator(box, device=dev)
    setup_s = time.perf_counter() - t0
    b = torch.as_tensor(rhs).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    for _ in range(max(warmup, 1)):
        x, rep = op.solve_device(b, tol=TOL, maxiter=20000)
        op.apply(b, "A")
    ms, ams = [], []
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        x, rep = op.solve_device(b, tol=TOL, maxiter=20000)
        ms.append(float(rep.elapsed_ms))
        flush.fill_(1.0)
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        op.apply(b, "A")
        e1.record()
        torch.cuda.synchronize(dev)
        ams.append(e0.elapsed_time(e1))
    N = box.n_red
    # algorithmic bytes of one apply: p read, y written, and the four pass
    # buffers each written once and read once (x pass writes U1 U2, y pass
    # reads them and writes V1 V2, z pass reads V1 V2)
    bytes_apply = 8.0 * N * (1 + 1 + 2 * 4)
    hbm, hbm_kind = peaks()
    am = float(np.median(ams))
    op.close()
    return {
        "workload": f"tensor cut box p={p} n={n} fractions (0.6,0.6,0.6), weak-penalty Poisson, Kronecker operator",
        "n_red": N, "iterations": int(rep.iterations), "converged": bool(rep.status == 0),
        "s_per_solve": float(np.mean(ms)) / 1e3, "apply_us": am * 1e3, "setup_s": setup_s,
        "roofline_apply": {"bound": "hbm", "kernel": "apply_kernel<KronOp>",
                           "achieved": bytes_apply / (am * 1e-3) / 1e9, "peak": hbm, "unit": "GB/s",
                           "frac": bytes_apply / (am * 1e-3) / 1e9 / hbm, "peak_kind": hbm_kind,
                           "algorithmic_bytes": bytes_apply, "traffic": NCU_TRAFFIC.get(("cut-box", n, p))},
    }


def run_cutbox_line(args, rank, world, local):
    """``--workload cut-box``: the tensor cut-box solve as its own line (one
    replica per rank; each rank solves its own copy)."""
    import torch

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    r = run_cutbox(args, dev, args.steps, n=args.cutbox_n, p=args.p, warmup=args.warmup)
    line = {"metric": "seconds per tensor cut-box Poisson solve (matrix-free Jacobi-PCG to 1e-9)",
            "value": r["s_per_solve"], "unit": "s/solve", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["s_per_solve"] * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "manufactured forcing u = exp(0.6x) cos(pi y) sin(pi z)",
            "config": {"workload": r["workload"], "n_red": r["n_red"], "iterations": r["iterations"],
                       "converged": r["converged"], "apply_us": r["apply_us"], "setup_s": r["setup_s"],
                       "l2": "flushed between timed launches", "parallelism": f"replicas x{world}"},
            "gpu_launches": args.steps * 2, "roofline": r["roofline_apply"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def extras_summary(args, rank, world, local):
    """Driver-measured summaries of the other hot-path workloads, run in the
    default invocation at few steps: the 72-system batch, the hill fast step
    and the tensor cut-box solve (each also has its own --workload line)."""
    import copy

    import torch

    dev = torch.device("cuda", local)
    sub = copy.copy(args)
    sub.steps, sub.warmup = min(args.steps, 5), min(args.warmup, 3)
    out = {}
    bl = run_batch(sub, rank, world, local, emit=False)
    out["batch"] = {k: bl[k] for k in ("metric", "value", "unit", "ms_per_step", "e2e")}
    out["batch"].update({"sequential_solves_per_s": bl["sequential"]["solves_per_s"],
                         "all_converged": bl["config"]["all_converged"], "autotuned": bl["config"]["autotuned"],
                         "roofline_frac": bl["roofline"]["frac"], "workload": bl["config"]["workload"]})
    hl = run_hill_step(sub, rank, world, local, emit=False)
    out["hill_step"] = {k: hl[k] for k in ("metric", "value", "unit", "data")}
    out["hill_step"].update({"workload": hl["config"]["workload"], "advect_ms": hl["config"]["advect_ms"],
                             "roofline": hl["roofline"], "divergence": hl["config"]["divergence"],
                             "setup_s": hl["config"]["setup_s"], "fastdiag_build": hl["config"]["fastdiag_build"]})
    out["cut_box"] = run_cutbox(args, dev, sub.steps, n=args.cutbox_n, warmup=sub.warmup)
    return out


if __name__ == "__main__":
    sys.exit(main())
