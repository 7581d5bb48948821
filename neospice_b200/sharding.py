"""Multi-GPU partitioning of independent circuit instances.

Instances never exchange data, so N GPUs split a batch with no collective on
the data path: each rank builds and solves its own share, and the only
communication is one reduction of the timings (and optionally a gather of the
per-instance results) after the timed region.

* ``partition(costs, world)``: a fixed global batch split across ranks by
  longest-processing-time-first greedy assignment on the estimated cost of
  each instance (e.g. nnz_LU x Newton iterations), so the slowest rank -- the
  one that sets the job's time -- carries as little as possible.
* ``rank_seed(seed, rank)``: the seed of rank r's own instances under weak
  scaling (every rank generates its own batch of the same size).
* ``max_over_ranks(values)``: the element-wise maximum across ranks of a few
  host doubles (timings), via torch.distributed on whatever backend the
  process group uses (NCCL on GPUs, gloo on CPU).
* ``run_partitioned(costs, run)``: strong scaling of a fixed global batch:
  this rank runs ``run(indices)`` on its share and every rank receives all
  results in global instance order (one gather after the work).
* ``dc_solve_global(circuits, costs)``: the batched DC operating point of a
  fixed global list of circuits split across the process group's ranks,
  each rank solving its share on its own GPU.
"""
from __future__ import annotations

import heapq


def partition(costs, world: int):
    """Instance indices per rank, greedy longest-first onto the least-loaded
    rank (ties to the lowest rank); every index appears exactly once."""
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


def rank_seed(seed: int, rank: int) -> int:
    return seed + 1000003 * rank


def max_over_ranks(values):
    """Element-wise max over ranks of a list of floats (identity when no
    process group is initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    backend = dist.get_backend()
    dev = "cuda" if backend == "nccl" else "cpu"
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def run_partitioned(costs, run):
    """Run a fixed global batch across the process group: this rank calls
    ``run(indices)`` on its share of ``partition(costs, world)`` (a list of
    per-instance results, in the order of ``indices``), and the results of
    every rank are gathered (all_gather_object, host objects) into one list
    in global instance order, returned on every rank.  Without a process
    group (or with one rank) it is ``run(range(len(costs)))``."""
    import torch.distributed as dist
    n = len(costs)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(run(list(range(n))))
    world, rank = dist.get_world_size(), dist.get_rank()
    mine = partition(costs, world)[rank]
    local = list(run(mine)) if mine else []
    if len(local) != len(mine):
        raise ValueError("run returned a result count different from its indices")
    gathered = [None] * world
    dist.all_gather_object(gathered, (mine, local))
    out = [None] * n
    for idx, res in gathered:
        for i, r in zip(idx, res):
            out[i] = r
    return out


def dc_solve_global(circuits, costs=None, symbolic=None):
    """Operating points of a fixed global list of finalized circuits split
    across the ranks (each rank solves its share as one DcBatch on its
    current GPU); returns, on every rank, a list of (solution as a numpy
    array, status, Newton iterations) in global order.  ``costs`` default to
    each circuit's nnz (a proxy for its LU work)."""
    import torch
    from .circuit import DcBatch
    if costs is None:
        costs = [float(c.info()["nnz"]) for c in circuits]

    def run(indices):
        batch = DcBatch([circuits[i] for i in indices],
                        symbolic=DcBatch.PER_INSTANCE if symbolic is None else symbolic)
        sols, status, iters = batch.run()
        torch.cuda.synchronize()
        st, it = status.cpu().numpy(), iters.cpu().numpy()
        return [(s.cpu().numpy() if hasattr(s, "cpu") else s, int(st[k]), int(it[k]))
                for k, s in enumerate(batch.split(sols))]

    return run_partitioned(costs, run)
