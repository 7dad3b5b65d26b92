"""Slices across GPUs: one process per GPU, independent slices, no data-path collective.

The reference's only parallelism is a process pool over independent slices
(algorithms/art.py:289, sir.py:260).  Here each rank takes a share of the
slices chosen by greedy longest-processing-time (LPT) on the per-slice cost
``n_op^2 * na`` (the projector's pixel x angle updates), reconstructs its share
in one batched plan, and the only communication is the optional gather of the
results to rank 0 at the end (host side, any torch.distributed backend).

  parts = lpt_partition(costs, world)         # same on every rank
  mine = parts[rank]                          # indices into the slice list
  ...reconstruct slices `mine`...
  full = gather_to_root(results, mine, n)     # rank 0: list of n results
"""
from __future__ import annotations

import heapq


def lpt_partition(costs, world: int):
    """Greedy LPT: slices in decreasing cost, each to the currently least-loaded rank.

    Deterministic (ties broken by slice index, then rank), so every rank
    computes the same partition without communicating.  Returns ``world``
    lists of slice indices, each in increasing order.
    """
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(p) for p in parts]


def loads(costs, parts):
    """Total cost per rank of a partition."""
    return [sum(float(costs[i]) for i in p) for p in parts]


def slice_cost(n_op: int, na: int) -> float:
    """Pixel x angle updates of one projector application on one slice."""
    return float(n_op) * n_op * na


def gather_to_root(results, indices, n_total: int, group=None):
    """Gathers each rank's ``results`` (one picklable object per index in
    ``indices``) to the group's first rank (rank 0 within ``group``) and
    returns them in slice order there (None on the other ranks).  A host-side
    gather: the only collective of the path."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        out = [None] * n_total
        for i, r in zip(indices, results):
            out[i] = r
        return out
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    payload = list(zip(indices, results))
    got = [None] * world if rank == 0 else None
    # gather_object takes the destination as a global rank
    dst = 0 if group is None else dist.get_global_rank(group, 0)
    dist.gather_object(payload, got, dst=dst, group=group)
    if rank != 0:
        return None
    out = [None] * n_total
    for part in got:
        for i, r in part:
            out[i] = r
    return out


def max_over_ranks(value: float, group=None) -> float:
    """The maximum of a per-rank scalar (e.g. a device-timed step) over all ranks."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64)
    backend = dist.get_backend(group)
    if backend == "nccl":
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
