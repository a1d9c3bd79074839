"""Batched persistent Jacobi-PCG over many uneven SPD systems (one launch).

The reference solves a sweep of systems one at a time, each through
``solve_spd`` / ``solve_cpu_cg`` / ``solve_gpu_cg``
(code/fast_solver_workbench.py:169-176, code/fast_solver_backends.py:90-132,
194-289).  Here all systems of a sweep go to the device together and are
solved by one persistent, graph-captured launch (``cutcell_batch_*`` in
libcutcell_b200.so): a team of 1-8 CTAs (a thread-block cluster) per system,
teams claiming systems heaviest first.  Per system the algorithm, stopping
test and report are those of ``solve_spd`` with plain FP64 Jacobi-PCG.

Tiles are chosen by a measuring autotuner (``BatchSolver.autotune``): cluster
size, shared-memory staging of the CSR slices, threads per CTA and lanes per
row are searched coordinate-wise by timing the real batch; the claim order
follows the measured cost (nonzeros x iterations) of the previous solve.

``partition_lpt`` splits a batch across GPUs (one process per GPU): systems
are independent, so there is no collective on the data path.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace
from time import perf_counter

import numpy as np

from . import _lib
from .fast_solver_backends import SolverReport, _report_from, as_csr

SMEM_OPTIN = 232448  # per-CTA opt-in shared memory on B200 (227 KB)
SMEM_PER_SM = 233472  # per-SM shared memory (228 KB)
_STATIC_SMEM = 512  # static shared memory of the kernel, rounded up
_SLOTS = 8 * 5 * 3 * 16  # reduction slots (5 groups x 3 values x 16 ranks)
_RESERVED_PER_CTA = 1024  # shared memory the runtime reserves per resident CTA


@dataclass(frozen=True)
class BatchConfig:
    cluster: int = 1  # CTAs per team (thread-block cluster): 1, 2, 4, 8 or 16
    threads: int = 256  # threads per CTA
    staging: str = "full"  # "none": CSR read from global; "full": one CTA per SM; "half": two per SM
    nnz_per_lane: int = 8  # target nonzeros per lane of a row group
    teams: int = 0  # 0 = as many as fit


def _vec_bytes(n: int) -> int:
    return 8 * ((n + 1) & ~1)


def fixed_smem(n_max: int, cluster: int) -> int:
    """Shared-memory bytes per CTA besides the staged matrix: full p and z, four
    row-slice vectors and the reduction slots (the kernel's BatchSmem)."""
    rows = -(-n_max // cluster)
    return 2 * _vec_bytes(n_max) + 4 * _vec_bytes(rows) + _SLOTS


def staging_bytes(cfg: BatchConfig, n_max: int, optin: int = SMEM_OPTIN, per_sm: int = SMEM_PER_SM) -> int:
    """Matrix budget per CTA for a staging mode (multiple of 16, >= 0)."""
    fixed = fixed_smem(n_max, cfg.cluster)
    if cfg.staging == "none":
        return 0
    if cfg.staging == "full":
        cap = optin - _STATIC_SMEM - fixed
    elif cfg.staging == "half":
        cap = per_sm // 2 - _RESERVED_PER_CTA - _STATIC_SMEM - fixed
    else:
        raise ValueError(f"unknown staging {cfg.staging!r}")
    return max(0, cap // 16 * 16)


def lanes_per_row(n: np.ndarray, nnz: np.ndarray, nnz_per_lane: int, threads: int = 256) -> np.ndarray:
    """Lanes per CSR row: the power of two nearest below mean-row-nnz /
    nnz_per_lane, clamped to [1, min(32, threads)]."""
    mean = np.asarray(nnz, dtype=float) / np.maximum(np.asarray(n, dtype=float), 1.0)
    want = np.maximum(mean / float(nnz_per_lane), 1.0)
    lanes = 2 ** np.floor(np.log2(want)).astype(np.int64)
    return np.clip(lanes, 1, min(32, threads)).astype(np.int32)


def claim_order(costs) -> np.ndarray:
    """Heaviest first; equal costs keep their input order."""
    c = np.asarray(costs, dtype=float)
    return np.argsort(-c, kind="stable").astype(np.int32)


def partition_lpt(costs, n_parts: int) -> list[list[int]]:
    """Longest-processing-time greedy: systems in decreasing cost, each to the
    currently lightest part (lowest index on ties).  Deterministic."""
    if n_parts < 1:
        raise ValueError("n_parts must be >= 1")
    load = [0.0] * n_parts
    parts: list[list[int]] = [[] for _ in range(n_parts)]
    for i in claim_order(costs):
        k = min(range(n_parts), key=lambda j: (load[j], j))
        parts[k].append(int(i))
        load[k] += float(costs[i])
    return [sorted(p) for p in parts]


@dataclass
class PackedSystems:
    n: np.ndarray  # int32 (m,)
    nnz: np.ndarray  # int32 (m,)
    indptr: np.ndarray  # int32, system i's n_i + 1 offsets back to back (relative)
    indices: np.ndarray  # int32, relative column indices
    data: np.ndarray  # float64
    vec_off: np.ndarray  # int64 (m + 1,), start of system i in packed vectors

    @property
    def count(self) -> int:
        return int(self.n.size)

    def split(self, v: np.ndarray) -> list[np.ndarray]:
        return [v[self.vec_off[i] : self.vec_off[i + 1]].copy() for i in range(self.count)]

    def pack(self, vs) -> np.ndarray:
        out = np.empty(int(self.vec_off[-1]))
        for i, v in enumerate(vs):
            v = np.asarray(v, dtype=float).ravel()
            if v.size != self.n[i]:
                raise ValueError(f"vector {i} has {v.size} entries, system has {self.n[i]}")
            out[self.vec_off[i] : self.vec_off[i + 1]] = v
        return out


def pack_systems(systems) -> PackedSystems:
    mats = [as_csr(A) for A in systems]
    for i, A in enumerate(mats):
        if A.shape[0] != A.shape[1]:
            raise ValueError(f"system {i} is not square")
        A.sort_indices()
    n = np.array([A.shape[0] for A in mats], dtype=np.int32)
    nnz = np.array([A.nnz for A in mats], dtype=np.int32)
    indptr = np.concatenate([A.indptr.astype(np.int32) for A in mats])
    indices = np.concatenate([A.indices.astype(np.int32) for A in mats]) if mats else np.zeros(0, np.int32)
    data = np.concatenate([A.data.astype(np.float64) for A in mats]) if mats else np.zeros(0)
    vec_off = np.concatenate([[0], np.cumsum(n.astype(np.int64))])
    return PackedSystems(n, nnz, indptr, indices, data, vec_off)


class BatchSolver:
    """Device-resident batch of SPD systems with its persistent-solve context."""

    def __init__(self, systems, device="cuda", config: BatchConfig | None = None):
        import torch

        self._lib = _lib.load()
        self.device = torch.device(device)
        self.packed = pk = pack_systems(systems)
        self.n_max = int(pk.n.max())
        self.indptr = torch.as_tensor(pk.indptr).to(self.device)
        self.indices = torch.as_tensor(pk.indices).to(self.device)
        self.data = torch.as_tensor(pk.data).to(self.device)
        self.rhs = torch.zeros(int(pk.vec_off[-1]), dtype=torch.float64, device=self.device)
        self.x = torch.zeros_like(self.rhs)
        self.costs = pk.nnz.astype(float) * np.sqrt(pk.n.astype(float))
        props = torch.cuda.get_device_properties(self.device)
        self.smem_optin = int(getattr(props, "shared_memory_per_block_optin", SMEM_OPTIN))
        self.smem_per_sm = int(getattr(props, "shared_memory_per_multiprocessor", SMEM_PER_SM))
        ctx = C.c_void_p()
        n_arr = np.ascontiguousarray(pk.n)
        z_arr = np.ascontiguousarray(pk.nnz)
        with torch.cuda.device(self.device):
            _lib.check(
                self._lib.cutcell_batch_create(
                    pk.count, n_arr.ctypes.data, z_arr.ctypes.data, self.indptr.data_ptr(), self.indices.data_ptr(),
                    self.data.data_ptr(), C.byref(ctx),
                ),
                "cutcell_batch_create",
            )
        self._ctx = ctx
        self.config: BatchConfig | None = None
        self.lanes = None
        self.order = None
        self.tuning: list[tuple[BatchConfig, float]] = []
        self.configure(config or BatchConfig())

    @property
    def count(self) -> int:
        return self.packed.count

    def configure(self, cfg: BatchConfig) -> None:
        import torch

        pk = self.packed
        lanes = lanes_per_row(pk.n, pk.nnz, cfg.nnz_per_lane, cfg.threads)
        order = claim_order(self.costs)
        c = _lib.CutcellBatchConfig(
            cfg.cluster, cfg.threads, staging_bytes(cfg, self.n_max, self.smem_optin, self.smem_per_sm), cfg.teams
        )
        with torch.cuda.device(self.device):
            _lib.check(
                self._lib.cutcell_batch_configure(self._ctx, C.byref(c), lanes.ctypes.data, order.ctypes.data),
                "cutcell_batch_configure",
            )
        self.config, self.lanes, self.order = cfg, lanes, order

    def info(self) -> dict:
        t, s = C.c_int32(), C.c_int32()
        _lib.check(self._lib.cutcell_batch_info(self._ctx, C.byref(t), C.byref(s)), "cutcell_batch_info")
        return {"teams": int(t.value), "smem_bytes": int(s.value)}

    def solve_device(self, rhs=None, x=None, *, tol=1e-8, maxiter=5000, preconditioner="jacobi"):
        """Solve all systems from the packed device rhs into the packed device x;
        returns the per-system CutcellReport array (the call waits)."""
        import torch

        rhs = self.rhs if rhs is None else rhs
        x = self.x if x is None else x
        if preconditioner not in ("none", "jacobi"):
            raise ValueError("batched solves support preconditioner 'none' or 'jacobi'")
        pre = _lib.PRECOND_JACOBI if preconditioner == "jacobi" else _lib.PRECOND_NONE
        reps = (_lib.CutcellReport * self.count)()
        with torch.cuda.device(self.device):
            st = self._lib.cutcell_batch_solve(
                self._ctx, rhs.data_ptr(), x.data_ptr(), float(tol), int(maxiter), pre, C.cast(reps, C.c_void_p),
                _lib.current_stream_ptr(),
            )
        if st not in (_lib.OK, _lib.E_SHAPE):
            _lib.check(st, "cutcell_batch_solve")
        return reps

    def timeline(self) -> dict:
        """Per-system start / end (microseconds from the first start) and team
        of the last solve, from the device global timer."""
        m = self.count
        t0, t1 = np.zeros(m), np.zeros(m)
        team = np.zeros(m, dtype=np.int32)
        _lib.check(
            self._lib.cutcell_batch_timeline(self._ctx, t0.ctypes.data, t1.ctypes.data, team.ctypes.data),
            "cutcell_batch_timeline",
        )
        return {"start_us": t0, "end_us": t1, "team": team}

    def learn_costs(self, reports) -> None:
        """Claim order from the measured work of a solve: nonzeros x iterations."""
        its = np.array([max(1, int(r.iterations)) for r in reports], dtype=float)
        self.costs = self.packed.nnz.astype(float) * its

    def autotune(self, *, tol=1e-9, maxiter=5000, preconditioner="jacobi", reps: int = 2, clusters=(1, 2, 4, 8, 16)):
        """Coordinate search over (cluster, staging), then threads, then lanes
        per row, timing the real batch on the current device rhs (device time
        of the captured solve, best of ``reps``).  Keeps the fastest."""
        first = self.solve_device(tol=tol, maxiter=maxiter, preconditioner=preconditioner)
        self.learn_costs(first)
        base = self.config or BatchConfig()

        def timed(cfg):
            try:
                self.configure(cfg)
            except _lib.CutcellLibraryError:
                return float("inf")
            best = float("inf")
            for _ in range(reps):
                r = self.solve_device(tol=tol, maxiter=maxiter, preconditioner=preconditioner)
                best = min(best, float(r[0].elapsed_ms))
            self.tuning.append((cfg, best))
            return best

        stage1 = [replace(base, cluster=c, staging=s) for c in clusters for s in ("none", "half", "full")]
        best = min(stage1, key=timed)
        stage2 = [replace(best, threads=t) for t in (128, 256, 512)]
        best = min(stage2, key=lambda c: timed(c) if c != best else self._time_of(c))
        stage3 = [replace(best, nnz_per_lane=k) for k in (4, 8, 16)]
        best = min(stage3, key=lambda c: timed(c) if c != best else self._time_of(c))
        self.configure(best)
        return best

    def _time_of(self, cfg) -> float:
        ts = [t for c, t in self.tuning if c == cfg]
        return min(ts) if ts else float("inf")

    def solve(self, rhs_list, *, tol=1e-8, maxiter=5000, preconditioner="jacobi"):
        """Host vectors in, host solutions and SolverReports out (one per system)."""
        import torch

        t0 = perf_counter()
        h = torch.from_numpy(self.packed.pack(rhs_list)).pin_memory()
        self.rhs.copy_(h, non_blocking=True)
        torch.cuda.synchronize(self.device)
        transfer = perf_counter() - t0
        tic = perf_counter()
        reps = self.solve_device(tol=tol, maxiter=maxiter, preconditioner=preconditioner)
        xs = self.packed.split(self.x.cpu().numpy())
        elapsed = perf_counter() - tic
        out = []
        for i in range(self.count):
            rep = _report_from(
                reps[i], backend="b200", method="b200-batched-pcg", preconditioner=preconditioner, precision="fp64",
                tol=tol, elapsed=elapsed, transfer=transfer,
            )
            out.append((xs[i], rep))
        return out

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.cutcell_batch_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_batch(
    systems, rhs, *, tol=1e-8, maxiter=5000, preconditioner="jacobi", device="cuda", autotune=False,
    config: BatchConfig | None = None,
) -> list[tuple[np.ndarray, SolverReport]]:
    """``solve_spd`` over a list of systems in one persistent launch: returns
    ``[(x_i, report_i)]`` in input order."""
    bs = BatchSolver(systems, device=device, config=config)
    try:
        if autotune:
            import torch

            bs.rhs.copy_(torch.from_numpy(bs.packed.pack(rhs)))
            bs.autotune(tol=tol, maxiter=maxiter, preconditioner=preconditioner)
        return bs.solve(rhs, tol=tol, maxiter=maxiter, preconditioner=preconditioner)
    finally:
        bs.close()


def solve_partitioned(systems, rhs, *, rank: int, world_size: int, costs=None, solve_fn=None, group=None, **kw):
    """Multi-GPU batch: one process per GPU, systems split by ``partition_lpt``
    (no data-path collective: the systems are independent).  Each rank solves
    its share with ``solve_fn`` (default ``solve_batch`` on the current
    device); the (index, x, report) results are then gathered on the host of
    every rank with ``all_gather_object``.  Returns the full result list in
    input order (every rank), or this rank's share when ``world_size == 1``."""
    import torch.distributed as dist

    systems = list(systems)
    if costs is None:
        pk = [as_csr(A) for A in systems]
        costs = [A.nnz * np.sqrt(A.shape[0]) for A in pk]
    parts = partition_lpt(costs, world_size)
    mine = parts[rank]
    fn = solve_fn or solve_batch
    res = fn([systems[i] for i in mine], [rhs[i] for i in mine], **kw) if mine else []
    local = [(i, x, r) for i, (x, r) in zip(mine, res)]
    if world_size == 1:
        gathered = [local]
    else:
        gathered = [None] * world_size
        dist.all_gather_object(gathered, local, group=group)
    out: list = [None] * len(systems)
    for part in gathered:
        for i, x, r in part:
            out[i] = (x, r)
    return out
