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
