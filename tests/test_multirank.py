"""The multi-GPU path's host side on CPU: two `gloo` ranks (world size 2).

bench.py shards rows by range (plain workloads: one range per rank; batched
and serving: ranges / requests round-robin) with no data-path collective; the
only collectives are the barrier and the whole-job reduction (max of timings,
sum of work).  Checked here: the shards are disjoint and cover the
configuration, and the reduction gives the max and the sum on every rank.
The column-shard workload gives every rank the same range instead; its
columns are split and gathered as tests/test_colshard.py checks.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shards = {}
        for name in ("plain-small", "plain-mid", "plain-top", "batched", "column-shard"):
            ranges, qcap, _ = bench.workload(name, rank, world)
            shards[name] = (ranges, qcap)
        reqs = bench.serving_requests(1, 32, 64.0, 2000)[rank::world]
        times, counts = bench.merge_over_ranks(dist, [1.0 + rank, 10.0 - rank], [100 * (rank + 1), 7], device="cpu")
        out = [None] * world
        dist.all_gather_object(out, (shards, reqs, times, counts))
        if rank == 0:
            q.put(out)
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_rank_main, args=(world, _free_port(), q), nprocs=world, start_method="spawn", join=True)
    out = q.get(timeout=60)
    (s0, r0, t0, c0), (s1, r1, t1, c1) = out
    # whole-job reduction, identical on both ranks
    assert t0 == t1 == [2.0, 10.0] and c0 == c1 == [300.0, 14.0]
    # plain workloads: consecutive disjoint ranges of the configured width
    a0, b0 = s0["plain-small"][0][0]
    a1, b1 = s1["plain-small"][0][0]
    assert (a0, b0 - a0) == (10**9, 10**6) and a1 == b0 and b1 - a1 == 10**6
    for name in ("plain-mid", "plain-top"):
        (x0, y0), = s0[name][0]
        (x1, y1), = s1[name][0]
        assert y0 <= x1 or y1 <= x0, name
        assert s0[name][1] == s1[name][1] == 2**32
    # column-shard: every rank holds the whole range, full search (its columns are split)
    assert s0["column-shard"] == s1["column-shard"] == ([(10**9, 10**9 + 10**6)], 0)
    # batched: the 256 ranges split round-robin, nothing lost or repeated
    import bench
    allr = bench.batched_ranges(0, max_width=2000)
    assert sorted(s0["batched"][0] + s1["batched"][0]) == sorted(allr)
    assert not set(s0["batched"][0]) & set(s1["batched"][0])
    # serving: requests split round-robin
    allq = bench.serving_requests(1, 32, 64.0, 2000)
    assert sorted(r0 + r1) == sorted(allq) and len(r0) == 16
