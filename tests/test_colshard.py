"""Column sharding (clwilson_b200.colshard) on CPU.

The planner: boundaries strictly increase from 2 to the first column above
every class target, with about equal modelled cells per piece once rank 0's
piece is charged the tail it also runs.

The flow: gloo ranks (world sizes 2 and 3) run search_columns_sharded with
an engine whose calls are answered by the oracle.  The pieces are products
over disjoint column intervals (oracle.range_product).  The row-wise product
uses exact integers, and the finishing call checks that its init is the
oracle's product over all columns.  Rank 0 must return the oracle's full
search: the same result lines and checksum.
"""
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from clwilson_b200 import colshard


def test_column_end_covers_every_target():
    for pmin, pmax in [(5, 6), (200, 564), (10**6, 10**6 + 3000), (10**13, 10**13 + 10**6)]:
        ps = oracle.list_primes(max(pmin, 5), min(pmax, pmin + 20000))
        end = colshard.column_end(pmax)
        for p in ps:
            p = int(p)
            T = (p - 1) // 6 if p % 3 == 1 else ((p - 1) // 4 if p % 12 == 5 else (p - 1) // 2)
            assert T < end
        assert end <= pmax // 2 + 1


@pytest.mark.parametrize("pmin,pmax,world", [(10**6, 10**6 + 3000, 2), (10**9, 10**9 + 10**6, 8),
                                             (1239053554603, 1239053554604, 4), ((1 << 62) - 10**6, (1 << 62) - 1, 8),
                                             (10**13, 10**13 + 10**6, 3)])
def test_pieces_balanced(pmin, pmax, world):
    b = colshard.column_pieces(pmin, pmax, world)
    assert len(b) == world + 1 and b[0] == 2 and b[-1] == colshard.column_end(pmax)
    assert all(x < y for x, y in zip(b, b[1:]))
    w = [colshard.modelled_cells(pmin, y) - colshard.modelled_cells(pmin, x) for x, y in zip(b, b[1:])]
    # rank 0 also runs the tail of every row: its piece is smaller by that
    extra = colshard.finish_cells(pmin, pmax)
    if extra > 1.0:
        assert w[0] < w[1]
    w[0] += extra
    assert max(w) <= 1.01 * min(w)
    # without the discount all pieces are equal
    b2 = colshard.column_pieces(pmin, pmax, world, rank0_extra=0.0)
    w2 = [colshard.modelled_cells(pmin, y) - colshard.modelled_cells(pmin, x) for x, y in zip(b2, b2[1:])]
    assert max(w2) <= 1.01 * min(w2)


def test_pieces_tiny_ranges():
    # fewer columns than ranks: one piece per column interval of length >= 1
    for pmin, pmax in [(5, 6), (5, 8), (7, 20), (200, 564)]:
        end = colshard.column_end(pmax)
        for world in (1, 2, 3, 8, 64):
            b = colshard.column_pieces(pmin, pmax, world)
            assert b[0] == 2 and b[-1] == end
            assert len(b) - 1 == max(1, min(world, end - 2))
            assert all(x < y for x, y in zip(b, b[1:]))
    with pytest.raises(ValueError):
        colshard.column_pieces(10**6, 10**6 + 10, 0)


class OracleEngine:
    """The engine calls of the sharded flow, answered by the oracle."""

    def __init__(self):
        self.finished = None

    @staticmethod
    def _class_targets(pmin, pmax):
        rows, targets = oracle.search(pmin, pmax, qcap=2)
        return rows, targets

    def rows_from(self, pmin, pmax, q_lo, q_cap=0, init=None):
        assert q_cap > q_lo >= 2 and init is None
        rows, targets = self._class_targets(pmin, pmax)
        for r in rows:
            r["s0"], r["s1"] = oracle.range_product(int(r["p"]), targets[int(r["type"])], q_lo, q_cap)
        return rows, None

    def rows_product(self, parts):
        out = parts[0].copy()
        for i in range(out.size):
            p = int(out["p"][i])
            v = 1
            for x in parts:
                assert int(x["p"][i]) == p
                v = v * (int(x["s0"][i]) + p * int(x["s1"][i])) % (p * p)
            out["s0"][i], out["s1"][i] = v % p, v // p
        return out

    def search_from(self, pmin, pmax, q_lo, init=None):
        want, targets = oracle.search(pmin, pmax, qcap=q_lo)
        assert q_lo > max(targets)
        assert np.array_equal(init["p"], want["p"])
        assert np.array_equal(init["s0"], want["s0"]) and np.array_equal(init["s1"], want["s1"])
        full, _ = oracle.search(pmin, pmax)
        self.finished = q_lo
        return SimpleNamespace(lines=oracle.result_lines(full), checksum=oracle.checksum(full))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, ranges, q):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from clwilson_b200 import colshard as cs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out = []
        for pmin, pmax in ranges:
            eng = OracleEngine()
            res = cs.search_columns_sharded(eng, pmin, pmax, rank, world)
            out.append(None if res is None else (res.lines, res.checksum, eng.finished))
        if rank == 0:
            q.put(out)
        else:
            assert all(x is None for x in out)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_flow_matches_oracle(world):
    ranges = [(200, 564), (10**6, 10**6 + 3000), (5, 8)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_rank_main, args=(world, _free_port(), ranges, q), nprocs=world, start_method="spawn",
                       join=True)
    got = q.get(timeout=60)
    for (pmin, pmax), (lines, ck, fin) in zip(ranges, got):
        full, _ = oracle.search(pmin, pmax)
        assert lines == oracle.result_lines(full) and ck == oracle.checksum(full)
        assert fin == colshard.column_end(pmax)
    # self-test case 5 (cl_wilson.cpp:2075-2081): 57 lines, checksum 00000000000080A3
    assert "%016X" % got[0][1] == "00000000000080A3" and len(got[0][0]) == 57
