"""Multi-rank host logic on CPU (gloo, world size 2): disjoint LPT shards that
cover the batch, weak-scaling seeds, max-over-ranks timing and summed counts."""
from __future__ import annotations

import os

import numpy as np
import torch.multiprocessing as mp

from prrtc_b200.shard import lpt_partition, weak_scaling_seeds


def test_lpt_partition_covers_and_balances():
    rng = np.random.default_rng(0)
    costs = rng.uniform(1, 100, 512)
    parts = lpt_partition(costs, 8)
    allidx = np.concatenate(parts)
    assert sorted(allidx.tolist()) == list(range(512))
    loads = [costs[p].sum() for p in parts]
    assert max(loads) <= costs.sum() / 8 + costs.max()


def test_weak_scaling_seeds_disjoint():
    a, b = set(weak_scaling_seeds(512, 0)), set(weak_scaling_seeds(512, 1))
    assert not a & b and len(a) == 512


def _worker(rank, world, port, q):
    import torch.distributed as dist

    from prrtc_b200.shard import lpt_partition, reduce_timing

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = np.arange(1, 41, dtype=np.float64)
        mine = lpt_partition(costs, world)[rank]
        secs, solved = reduce_timing(1.0 + rank, len(mine))
        dist.barrier()
        q.put((rank, mine.tolist(), secs, solved))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 1000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    assert sorted(out[0][1] + out[1][1]) == list(range(40))
    assert all(o[2] == 2.0 for o in out)        # max of 1.0, 2.0
    assert all(o[3] == 40 for o in out)         # all problems counted once


def test_strong_split_shares_one_batch():
    """bench --split strong: the ranks' longest-processing-time shares of one
    common batch are disjoint and cover it."""
    import bench
    from conftest import oracle_checker

    shares = [bench.make_workload(16, r, oracle_checker, "strong", 2) for r in range(2)]
    seeds = [sorted(p.seed for p in s) for s in shares]
    assert not set(seeds[0]) & set(seeds[1])
    assert sorted(seeds[0] + seeds[1]) == list(range(100000, 100016))
    costs = [sum(bench.problem_cost(p) for p in s) for s in shares]
    assert max(costs) <= sum(costs) / 2 + max(bench.problem_cost(p) for s in shares for p in s)
