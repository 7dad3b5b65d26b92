"""CPU tests of the multi-rank slice sharding (sharding.py), world size 2 over gloo.

The GPU path shards independent slices across ranks with no data-path
collective; what the ranks share is the partition (computed identically on
each rank), the max-over-ranks step time and the final gather of results to
rank 0.  These run here as two gloo processes on 127.0.0.1.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from iterative_tomographic_reconstruction_algorithms_b200.sharding import (gather_to_root, loads,
                                                                           lpt_partition, max_over_ranks,
                                                                           slice_cost)


def _costs(n=512, seed=4):
    rng = np.random.default_rng(seed)
    sides = rng.choice([256, 512, 1024, 2048], size=n, p=[0.4, 0.3, 0.2, 0.1])
    return [slice_cost(int(np.ceil(1.5 * s)), int(round(1.5 * s))) for s in sides]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_lpt_partition_covers_and_balances(world):
    costs = _costs()
    parts = lpt_partition(costs, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(costs)))
    ld = loads(costs, parts)
    # LPT bound: max load <= mean + largest job
    assert max(ld) <= sum(costs) / world + max(costs) + 1e-6
    assert lpt_partition(costs, world) == parts  # deterministic


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = _costs(40, seed=9)
        parts = lpt_partition(costs, world)
        mine = parts[rank]
        # each rank "reconstructs" its slices: a value derived from the slice index
        results = [np.full(3, float(i) * 2.0) for i in mine]
        full = gather_to_root(results, mine, len(costs))
        t = max_over_ranks(10.0 + rank)
        if rank == 0:
            ok = all(full[i] is not None and float(full[i][0]) == 2.0 * i for i in range(len(costs)))
            q.put((ok, t, [len(p) for p in parts]))
        else:
            assert full is None
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_partition_gather_and_max():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    ok, t, sizes = q.get(timeout=10)
    assert ok
    assert t == 11.0
    assert sum(sizes) == 40


def _subgroup_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sub = dist.new_group([1, 2])            # a group without global rank 0
        if rank in (1, 2):
            costs = _costs(10, seed=3)
            parts = lpt_partition(costs, 2)
            mine = parts[rank - 1]
            full = gather_to_root([i * 3 for i in mine], mine, len(costs), group=sub)
            if rank == 1:                        # rank 0 within the group
                q.put(full == [i * 3 for i in range(len(costs))])
            else:
                assert full is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_gather_to_root_in_a_subgroup_without_global_rank_0():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_subgroup_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert q.get(timeout=10) is True


# ---------------------------------------------------------------------------
# One slice sharded by angles (AngleShardedProjector), over gloo on CPU.  The
# plan is a stand-in with the plans' row convention, built on the FP64
# oracle's projector one angle at a time: angle v's row is v (pd) or
# na - 1 - v (dd), the adjoint sums the angles' back-projections.
# ---------------------------------------------------------------------------
class _OraclePlan:
    KIND = {"pd": 0, "dd": 2}

    def __init__(self, kind, n, angles):
        from oracle.oracle import Oracle
        self.L = Oracle().L
        self.kind, self.n, self.angles = kind, n, np.asarray(angles, np.float32)
        self.reversed = kind == "dd"

    def _one(self, v, data, oper):
        import ctypes
        fp = ctypes.POINTER(ctypes.c_float)
        dp = ctypes.POINTER(ctypes.c_double)
        a = np.ascontiguousarray(self.angles[v:v + 1])
        data = np.ascontiguousarray(data, np.float32)
        out = np.zeros((1, self.n) if oper == 0 else (self.n, self.n), np.float64)
        getattr(self.L, f"orc_{self.kind}")(data.ctypes.data_as(fp), self.n, a.ctypes.data_as(fp), 1, oper,
                                            out.ctypes.data_as(dp))
        return out

    def forward(self, x):
        import torch
        na = len(self.angles)
        rows = np.zeros((na, self.n), np.float64)
        for v in range(na):
            rows[na - 1 - v if self.reversed else v] = self._one(v, x.numpy(), 0)[0]
        return torch.from_numpy(rows.astype(np.float32))

    def adjoint(self, y):
        import torch
        na = len(self.angles)
        img = np.zeros((self.n, self.n), np.float64)
        for v in range(na):
            img += self._one(v, y.numpy()[na - 1 - v if self.reversed else v][None, :], 1)
        return torch.from_numpy(img.astype(np.float32))


def _angle_worker(rank, world, port, kind, q):
    import torch
    import torch.distributed as dist

    from iterative_tomographic_reconstruction_algorithms_b200.sharding import AngleShardedProjector
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        n, na = 24, 17
        rng = np.random.default_rng(7)
        angles = np.sort(rng.uniform(0.05, 3.0, na)).astype(np.float32)
        x = torch.from_numpy(rng.standard_normal((n, n)).astype(np.float32))
        y = torch.from_numpy(rng.standard_normal((na, n)).astype(np.float32))
        sp = AngleShardedProjector(lambda a: _OraclePlan(kind, n, a), _OraclePlan.KIND[kind], angles)
        full = _OraclePlan(kind, n, angles)
        rows = sp.forward(x)
        gathered = sp.forward(x, gather=True)
        adj = sp.adjoint(y[sp.rows])
        ref_rows, ref_adj = full.forward(x), full.adjoint(y)
        ok = (torch.equal(rows, ref_rows[sp.rows]) and torch.equal(gathered, ref_rows)
              and float((adj - ref_adj).norm() / ref_adj.norm()) < 1e-6)
        q.put((rank, ok, sp.local))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind,world", [("dd", 2), ("pd", 2), ("dd", 3)])
def test_angle_sharded_slice_over_gloo(kind, world):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_angle_worker, args=(r, world, port, kind, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(world))
    assert all(ok for _, ok, _ in got)
    assert sum(local for _, _, local in got) == 17
