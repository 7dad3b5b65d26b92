"""Work across GPUs, one process per GPU.

Slices: independent slices, no data-path collective.

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

One huge slice: its angles (AngleShardedProjector).  Each rank holds a plan for
a contiguous range of the angles; the forward needs no communication (its rows
are a contiguous block of the full sinogram), and the adjoint's partial images
are summed by one all-reduce of 4 n^2 bytes.
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


# Radon kinds whose plans write angle v's projection to row na - 1 - v
# (radon_dd.c:79,181,273; radon_ss.c:111); the others write row v.
_REVERSED_ROWS = {2, 3}  # TOMO_KIND_DD, TOMO_KIND_SS


def angle_shards(na: int, world: int):
    """Contiguous angle ranges [start, stop), one per rank, as equal as the
    count allows (every angle of a Radon projector costs the same)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(na, world)
    out, start = [], 0
    for r in range(world):
        stop = start + base + (1 if r < extra else 0)
        out.append((start, stop))
        start = stop
    return out


class AngleShardedProjector:
    """One slice whose angles are split across the ranks of ``group``.

    ``make_plan(sub_angles)`` builds this rank's plan for its contiguous share
    of ``angles`` (an object with ``forward(x)`` and ``adjoint(y)`` on CUDA
    float32 tensors, e.g. ``_lib.Plan(kind, n, sub_angles)``); ``kind`` is the
    Radon kind (TOMO_KIND_PD / RD / DD / SS), which fixes where the plan puts
    each angle's row.

    ``forward(x)``: this rank's rows, which are the full sinogram's rows
    ``rows`` (a contiguous block); ``gather=True`` returns the full sinogram on
    every rank instead (one all-gather).  ``adjoint(y_rows)``: this rank's
    rows in, the full adjoint on every rank out: the partial images are summed
    by an all-reduce (NCCL's order, fixed for a given set of ranks, so
    deterministic; the sum is taken in another order than on one GPU, so equal
    to it up to rounding).  With no process group (or one rank) both are the
    plan's own results.
    """

    def __init__(self, make_plan, kind: int, angles, group=None):
        import torch.distributed as dist
        self.group = group
        self.dist = dist.is_available() and dist.is_initialized()
        self.rank = dist.get_rank(group) if self.dist else 0
        self.world = dist.get_world_size(group) if self.dist else 1
        angles = list(angles)
        self.na = len(angles)
        self.shards = angle_shards(self.na, self.world)
        start, stop = self.shards[self.rank]
        self.local = stop - start
        self.plan = make_plan(angles[start:stop]) if self.local > 0 else None
        # full-sinogram rows of this rank's rows: angle v's row is v, or na - 1 - v
        first = (self.na - stop) if int(kind) in _REVERSED_ROWS else start
        self.rows = slice(first, first + self.local)
        self.row_starts = [((self.na - b) if int(kind) in _REVERSED_ROWS else a) for a, b in self.shards]

    def forward(self, x, gather: bool = False):
        import torch
        n = x.shape[-1]
        mine = self.plan.forward(x) if self.plan is not None else torch.zeros(
            (0, n), dtype=torch.float32, device=x.device)
        mine = mine.reshape(self.local, n)
        if not gather:
            return mine
        full = torch.empty((self.na, n), dtype=torch.float32, device=x.device)
        if self.world == 1:
            full[self.rows] = mine
            return full
        import torch.distributed as dist
        # all-gather takes equal sizes: every block padded to the largest share
        m = max(b - a for a, b in self.shards)
        padded = torch.zeros((m, n), dtype=torch.float32, device=x.device)
        padded[:self.local] = mine
        parts = [torch.empty((m, n), dtype=torch.float32, device=x.device) for _ in self.shards]
        dist.all_gather(parts, padded, group=self.group)
        for (a, b), r0, part in zip(self.shards, self.row_starts, parts):
            full[r0:r0 + (b - a)] = part[:b - a]
        return full

    def adjoint(self, y_rows):
        import torch
        n = y_rows.shape[-1]
        if self.plan is not None:
            img = self.plan.adjoint(y_rows.reshape(self.local, n).contiguous()).reshape(n, n)
        else:
            img = torch.zeros((n, n), dtype=torch.float32, device=y_rows.device)
        if self.world > 1:
            import torch.distributed as dist
            dist.all_reduce(img, op=dist.ReduceOp.SUM, group=self.group)
        return img
