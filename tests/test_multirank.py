"""The N-rank path of bench.py on CPU: world_size 2 over gloo (127.0.0.1).
A single cloud runs as replicas, the batched workload is split by LPT over
the n log n cost estimate with no collective on the data path; the only
collectives are the barrier, the max of the ranks' times and the sum of their
point counts."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    import bench
    import torch.distributed as dist
    from wtet_b200 import synthetic as syn

    r, _, w = bench.dist_setup(world, backend="gloo")
    clouds = syn.batched_clouds(37, 5, lo=8, hi=64)
    mine = bench.shard(clouds, r, w)
    n_mine = sum(len(c) for c in mine)
    total = bench.reduce_over_ranks(float(n_mine), w, "sum", device="cpu")
    t = bench.reduce_over_ranks(float(10 + r), w, "max", device="cpu")
    single = bench.shard([clouds[0]], r, w)
    bench.barrier(w)
    out.put((r, [len(c) for c in mine], n_mine, total, t, len(single)))
    dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from wtet_b200 import synthetic as syn

    import bench

    clouds = syn.batched_clouds(37, 5, lo=8, hi=64)
    sizes = [len(c) for c in clouds]
    owner = bench.lpt_assign(sizes, world)
    # LPT partition: every cloud on exactly one rank, input order kept inside a rank
    assert res[0][1] == [s for s, o in zip(sizes, owner) if o == 0]
    assert res[1][1] == [s for s, o in zip(sizes, owner) if o == 1]
    assert sorted(res[0][1] + res[1][1]) == sorted(sizes)
    assert res[0][3] == res[1][3] == float(sum(sizes))   # summed point count on every rank
    assert res[0][4] == res[1][4] == 11.0                # max of the ranks' times
    assert res[0][5] == res[1][5] == 1                   # a single cloud is replicated, not split


def test_lpt_balances_the_batched_workload():
    """On the benchmark's 4,096 log-uniform clouds, LPT keeps every rank within
    1% of the mean estimated cost at 2, 4 and 8 ranks (round robin does not)."""
    import sys

    sys.path.insert(0, ROOT)
    import bench
    from wtet_b200 import synthetic as syn

    sizes = [int(s) for s in syn.batched_sizes(4096, 4)]
    cost = [bench.cloud_cost(s) for s in sizes]
    for world in (2, 4, 8):
        owner = bench.lpt_assign(sizes, world)
        load = np.zeros(world)
        for c, o in zip(cost, owner):
            load[o] += c
        assert load.max() / load.mean() < 1.01, (world, load)
    # deterministic
    assert bench.lpt_assign(sizes, 4) == bench.lpt_assign(sizes, 4)
