"""Host logic of the batched solve (CPU): lanes per row, claim order, LPT
partition, packing, staging budgets, and the two-rank partitioned solve over
gloo with a CPU stand-in for the device solve."""

from __future__ import annotations

import os

import numpy as np
import pytest
import scipy.sparse as sp

from cutcell_b200 import batch as bt


def _spd(n, seed, density=0.2):
    rng = np.random.default_rng(seed)
    M = sp.random(n, n, density=density, random_state=rng, format="csr")
    return sp.csr_matrix(M @ M.T + n * sp.eye(n))


def test_lanes_per_row_rule():
    n = np.array([10, 10, 10, 10, 100])
    nnz = np.array([10, 80, 500, 5000, 100 * 121])
    np.testing.assert_array_equal(bt.lanes_per_row(n, nnz, 8), [1, 1, 4, 32, 8])
    np.testing.assert_array_equal(bt.lanes_per_row(n, nnz, 4), [1, 2, 8, 32, 16])
    assert bt.lanes_per_row(n, nnz, 1, threads=16).max() == 16


def test_claim_order_is_stable_heaviest_first():
    np.testing.assert_array_equal(bt.claim_order([1.0, 5.0, 5.0, 2.0]), [1, 2, 3, 0])


def test_partition_lpt_balances_and_covers():
    rng = np.random.default_rng(3)
    costs = rng.uniform(1, 100, size=72)
    for k in (1, 2, 3, 8):
        parts = bt.partition_lpt(costs, k)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(72))
        loads = [costs[p].sum() for p in parts]
        # LPT bound: makespan <= (4/3 - 1/(3k)) OPT <= (4/3) max(mean, max cost) + max cost
        assert max(loads) <= max(sum(costs) / k, costs.max()) * 4.0 / 3.0 + 1e-9
        assert bt.partition_lpt(costs, k) == parts
    with pytest.raises(ValueError):
        bt.partition_lpt(costs, 0)


def test_pack_and_split_round_trip():
    systems = [_spd(n, s) for s, n in enumerate((5, 9, 1, 17))]
    pk = bt.pack_systems(systems)
    assert pk.count == 4
    assert list(pk.n) == [5, 9, 1, 17] and pk.indptr.size == sum(n + 1 for n in pk.n)
    off = 0
    for i, A in enumerate(systems):
        seg = pk.indptr[off : off + pk.n[i] + 1]
        assert seg[0] == 0 and seg[-1] == A.nnz
        off += pk.n[i] + 1
    vs = [np.arange(n, dtype=float) + 10 * i for i, n in enumerate(pk.n)]
    for a, b in zip(pk.split(pk.pack(vs)), vs):
        np.testing.assert_array_equal(a, b)
    with pytest.raises(ValueError):
        pk.pack([np.zeros(3)] * 4)


def test_staging_budgets_fit_shared_memory():
    for c in (1, 2, 4, 8, 16):
        for mode in ("none", "half", "full"):
            cfg = bt.BatchConfig(cluster=c, staging=mode)
            m = bt.staging_bytes(cfg, 841)
            assert m % 16 == 0 and m >= 0
            total = bt.fixed_smem(841, c) + m + bt._STATIC_SMEM
            assert total <= bt.SMEM_OPTIN
            if mode == "half":
                assert 2 * (total + bt._RESERVED_PER_CTA) <= bt.SMEM_PER_SM
    assert bt.staging_bytes(bt.BatchConfig(staging="none"), 841) == 0


def _cpu_solve(systems, rhs, **kw):
    from oracle.pcg import cg_loop

    out = []
    for A, b in zip(systems, rhs):
        x, rep = cg_loop(A, b, tol=kw.get("tol", 1e-9), maxiter=kw.get("maxiter", 5000))
        out.append((x, rep["iterations"]))
    return out


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        systems = [_spd(n, s) for s, n in enumerate((12, 30, 7, 25, 18, 3, 40))]
        rng = np.random.default_rng(11)
        rhs = [rng.standard_normal(A.shape[0]) for A in systems]
        out = bt.solve_partitioned(systems, rhs, rank=rank, world_size=world, solve_fn=_cpu_solve, tol=1e-10)
        err = max(np.linalg.norm(A @ x - b) / np.linalg.norm(b) for A, b, (x, _) in zip(systems, rhs, out))
        q.put((rank, len(out), float(err), sorted(bt.partition_lpt([A.nnz * np.sqrt(A.shape[0]) for A in systems], world)[rank])))
    finally:
        dist.destroy_process_group()


def test_partitioned_solve_two_ranks_gloo():
    import multiprocessing as mp
    import socket

    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    shares = [r[3] for r in res]
    assert sorted(shares[0] + shares[1]) == list(range(7)) and shares[0] and shares[1]
    for rank, count, err, _ in res:
        assert count == 7 and err < 1e-9
