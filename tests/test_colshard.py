"""Column sharding (clwilson_b200.colshard) on CPU.

The planner: boundaries strictly increase from 2 to the first column above
every class target, with about equal modelled work per piece once rank 0's
piece is charged the finish it also runs; the range model of narrow ranges
has the oracle's class counts and targets.

The flow: gloo ranks (world sizes 2 and 3) run search_columns_sharded with
an engine whose calls are answered by the oracle, also with the other ranks
planning different boundaries (rank 0's are broadcast).  The pieces are products
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


@pytest.mark.parametrize("pmin,pmax,world", [(10**6, 10**6 + 3000, 2), (10**6, 10**6 + 3000, 5),
                                             (10**9, 10**9 + 10**6, 8),
                                             (1239053554603, 1239053554604, 4), ((1 << 62) - 10**6, (1 << 62) - 1, 8),
                                             (10**13, 10**13 + 10**6, 3)])
def test_pieces_balanced(pmin, pmax, world):
    m = colshard.RangeModel(pmin, pmax)
    b = colshard.column_pieces(pmin, pmax, world, model=m)
    assert len(b) == world + 1 and b[0] == 2 and b[-1] == colshard.column_end(pmax)
    assert all(x < y for x, y in zip(b, b[1:]))
    w = [m.work(y) - m.work(x) for x, y in zip(b, b[1:])]
    # rank 0 also runs the finish: its piece is smaller by the modelled finish,
    # or one column when the finish outweighs a whole piece
    assert w[0] < w[1]
    if m.finish() < m.work(b[-1]) / world:
        w[0] += m.finish()
    else:
        assert b[1] == 3
        w = w[1:]
    assert max(w) <= 1.01 * min(w)
    # without the discount all pieces are equal
    b2 = colshard.column_pieces(pmin, pmax, world, rank0_extra=0.0, model=m)
    w2 = [m.work(y) - m.work(x) for x, y in zip(b2, b2[1:])]
    assert max(w2) <= 1.01 * min(w2)


def test_range_model_exact_for_narrow_ranges():
    # class counts and shared targets as the oracle finds them
    for pmin, pmax in [(200, 564), (10**6, 10**6 + 3000), (2**31 - 1000, 2**31 + 1000), (10**12, 10**12 + 5000)]:
        m = colshard.RangeModel(pmin, pmax)
        rows, targets = oracle.search(pmin, pmax, qcap=2)
        assert m.rows == len(rows)
        assert list(m.targets) == [int(t) for t in targets]
        counts = np.bincount(rows["type"].astype(np.int64), minlength=3)
        assert np.allclose(np.array(m.share) * len(rows), counts)
    # self-test case 1: one class-0 prime; every boundary but the end lies below its target
    m = colshard.RangeModel(1239053554603, 1239053554604)
    assert m.rows == 1 and m.share == (1.0, 0.0, 0.0) and m.targets == ((1239053554603 - 1) // 6, 0, 0)
    b = colshard.column_pieces(1239053554603, 1239053554604, 3, model=m)
    assert all(x < m.targets[0] for x in b[:-1])
    # wide ranges: asymptotic shares, targets (pmin - 1) / k
    m = colshard.RangeModel(10**9, 10**9 + 10**6)
    assert m.share == colshard.CLASS_SHARE and abs(m.rows - 10**6 / np.log(10**9)) < 1


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
        assert q_cap >= q_lo >= 2 and init is None
        rows, targets = self._class_targets(pmin, pmax)
        for r in rows:
            if q_cap == q_lo:                      # no column: the empty product
                r["s0"], r["s1"] = 1, 0
            else:
                r["s0"], r["s1"] = oracle.range_product(int(r["p"]), targets[int(r["type"])], q_lo, q_cap)
        return rows, None

    def rows_product(self, parts, p=None):
        # gathered pieces arrive as (n, 2) digit arrays, 16 bytes per row
        assert p is not None
        assert all(x.shape == (len(p), 2) and x.dtype == np.uint64 for x in parts)
        out = np.zeros(len(p), dtype=oracle.ROW_DTYPE)
        out["p"] = p
        for i in range(out.size):
            q = int(p[i])
            v = 1
            for x in parts:
                v = v * (int(x[i, 0]) + q * int(x[i, 1])) % (q * q)
            out["s0"][i], out["s1"][i] = v % q, v // q
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


def _rank_main(rank, world, port, ranges, q, perturb=False, own_gather=False):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist
    from clwilson_b200 import colshard as cs
    if perturb and rank > 0:
        # this rank would plan other boundaries; rank 0's broadcast ones must win
        plan = cs.column_pieces
        cs.column_pieces = lambda lo, hi, w, **k: [b if i in (0, len(bs) - 1) else b + 1 + i
                                                   for bs in [plan(lo, hi, w, **k)] for i, b in enumerate(bs)]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out = []
        # a caller's gather: no broadcast of rank 0's boundaries, so with
        # perturbed plans rank 0 must find the mismatch in the pieces' headers
        gather = (lambda arr: cs.gather_to_rank0(arr, rank, world)) if own_gather else None
        for pmin, pmax in ranges:
            eng = OracleEngine()
            try:
                res = cs.search_columns_sharded(eng, pmin, pmax, rank, world, gather=gather)
            except ValueError as e:
                assert rank == 0
                out.append(("raised", str(e)))
                continue
            out.append(None if res is None else (res.lines, res.checksum, eng.finished))
        if rank == 0:
            q.put(out)
        else:
            assert all(x is None for x in out)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,perturb", [(2, False), (3, False), (3, True)])
def test_sharded_flow_matches_oracle(world, perturb):
    ranges = [(200, 564), (10**6, 10**6 + 3000), (5, 8)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_rank_main, args=(world, _free_port(), ranges, q, perturb), nprocs=world,
                       start_method="spawn", join=True)
    got = q.get(timeout=60)
    for (pmin, pmax), (lines, ck, fin) in zip(ranges, got):
        full, _ = oracle.search(pmin, pmax)
        assert lines == oracle.result_lines(full) and ck == oracle.checksum(full)
        assert fin == colshard.column_end(pmax)
    # self-test case 5 (cl_wilson.cpp:2075-2081): 57 lines, checksum 00000000000080A3
    assert "%016X" % got[0][1] == "00000000000080A3" and len(got[0][0]) == 57


@pytest.mark.parametrize("perturb", [False, True])
def test_sharded_flow_with_own_gather(perturb):
    # a caller-supplied gather (here the tensor gather, called directly):
    # agreeing plans give the oracle's result; when the other ranks plan other
    # boundaries, rank 0 refuses the pieces instead of multiplying them
    world = 3
    ranges = [(200, 564), (10**6, 10**6 + 3000)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    mp.start_processes(_rank_main, args=(world, _free_port(), ranges, q, perturb, True), nprocs=world,
                       start_method="spawn", join=True)
    got = q.get(timeout=60)
    for (pmin, pmax), r in zip(ranges, got):
        if perturb:
            assert r[0] == "raised" and "column pieces disagree" in r[1]
        else:
            full, _ = oracle.search(pmin, pmax)
            assert r[0] == oracle.result_lines(full) and r[1] == oracle.checksum(full)


def test_piece_headers():
    b = [2, 100, 5000, 9001]
    rows = np.zeros(3, dtype=oracle.ROW_DTYPE)
    rows["s0"], rows["s1"] = [1, 2, 3], [4, 5, 6]
    parts = [colshard.piece_digits(rows, colshard.piece_interval(b, r)) for r in range(4)]
    assert parts[0].shape == (4, 2) and tuple(parts[0][0]) == (2, 100) and tuple(parts[3][0]) == (0, 0)
    got = colshard.check_pieces(b, parts)
    assert len(got) == 3 and all(np.array_equal(x[:, 0], [1, 2, 3]) for x in got)
    parts[1][0, 1] += 1
    with pytest.raises(ValueError):
        colshard.check_pieces(b, parts)
