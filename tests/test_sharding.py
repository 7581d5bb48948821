"""Multi-rank host logic on CPU (gloo, world size 2): instance partitioning
covers every instance exactly once and balances the estimated cost, ranks
generate distinct weak-scaling batches, the timing reduction returns the
maximum over ranks on every rank, and a partitioned fixed batch gathers
every rank's results in global order on every rank."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

from neospice_b200 import sharding


def test_partition_covers_and_balances():
    rng = np.random.default_rng(3)
    costs = rng.lognormal(0.0, 1.0, 1000)
    for world in (1, 2, 3, 8):
        parts = sharding.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        # LPT bound: max load <= mean + largest single cost
        assert max(loads) <= sum(loads) / world + costs.max() + 1e-9


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from neospice_b200 import workloads
        seed = sharding.rank_seed(0, rank)
        meshes = workloads.diode_mesh_batch(6, seed=seed, side_range=(4, 8))
        sizes = [m.side for m in meshes]
        # each rank's stand-in for its device time; the job time is the max
        mx = sharding.max_over_ranks([1.0 + rank, 10.0 - rank])
        parts = sharding.partition([float(s * s) for s in range(20)], world)
        # strong scaling of a fixed batch: each rank runs its share, all
        # results come back in global order on every rank
        gathered = sharding.run_partitioned([float(s * s) for s in range(20)],
                                            lambda idx: [(i * i, rank) for i in idx])
        out.put((rank, sizes, mx, parts[rank], gathered))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (_, s0, m0, p0, g0), (_, s1, m1, p1, g1) = res
    assert s0 != s1                      # distinct per-rank batches
    assert m0 == m1 == [2.0, 10.0]       # max over ranks, on both ranks
    assert sorted(p0 + p1) == list(range(20))
    assert g0 == g1                      # the gathered results, on both ranks
    assert [v for v, _ in g0] == [i * i for i in range(20)]
    assert [r for _, r in g0] == [0 if i in p0 else 1 for i in range(20)]
