"""The N-rank path of bench.py on CPU: world_size 2 over gloo (127.0.0.1).
A single cloud runs as replicas, the batched workload is split round robin
with no collective on the data path; the only collectives are the barrier,
the max of the ranks' times and the sum of their point counts."""
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

    clouds = syn.batched_clouds(37, 5, lo=8, hi=64)
    sizes = [len(c) for c in clouds]
    # round robin partition: every cloud on exactly one rank
    assert res[0][1] == sizes[0::2] and res[1][1] == sizes[1::2]
    assert res[0][3] == res[1][3] == float(sum(sizes))   # summed point count on every rank
    assert res[0][4] == res[1][4] == 11.0                # max of the ranks' times
    assert res[0][5] == res[1][5] == 1                   # a single cloud is replicated, not split
