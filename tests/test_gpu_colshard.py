"""Column sharding on one GPU, with the ranks' pieces run one after another.

* wl_rows_product against exact integer products, for primes of every limb
  width (2, 3 and 4 32-bit limbs) and one to five parts.
* The sharded search must equal the one-call wl_search of the same range:
  pieces from wl_rows_from starting at 1, their row-wise product, then the
  finishing wl_search_from.  Result lines, checksum and the product rows are
  compared, with the pieces as rows and as the 16-byte digit arrays ranks
  exchange.  Ranges: self-test case 5, rows straddling 2^31, a 20,000-wide
  range cut into 8 pieces, and self-test case 1, whose columns reach 2.07e11:
  its pieces start above 2^32 or hold no column of the row at all.
"""
import random

import numpy as np
import pytest

import clwilson_b200 as wl
import oracle
from clwilson_b200 import colshard

pytestmark = pytest.mark.gpu


def _rows(ps, digits):
    r = np.zeros(len(ps), dtype=wl.ROW_DTYPE)
    r["p"] = ps
    r["s0"] = [d[0] for d in digits]
    r["s1"] = [d[1] for d in digits]
    return r


@pytest.mark.parametrize("nparts", [1, 2, 5])
def test_rows_product_exact(engine, nparts):
    rng = random.Random(1000 + nparts)
    ps = [int(x) for x in oracle.list_primes(5, 200)]
    for lo, hi in [(2**31 - 300, 2**31 + 300), (2**47 - 3000, 2**47 + 3000), (2**62 - 4000, 2**62 - 1)]:
        ps += [int(x) for x in oracle.list_primes(lo, hi)][:40]
    parts = []
    for _ in range(nparts):
        digs = []
        for p in ps:
            d = (rng.randrange(p), rng.randrange(p))
            if rng.random() < 0.05:
                d = (p - 1, p - 1)             # the largest value, p^2 - 1
            digs.append(d)
        parts.append(_rows(ps, digs))
    got = engine.rows_product(parts)
    for i, p in enumerate(ps):
        v = 1
        for x in parts:
            v = v * (int(x["s0"][i]) + p * int(x["s1"][i])) % (p * p)
        assert (int(got["s0"][i]), int(got["s1"][i])) == (v % p, v // p), p


def test_rows_product_rejects_bad_digits(engine):
    good = _rows([7, 11], [(1, 2), (3, 4)])
    bad = _rows([7, 11], [(7, 0), (3, 4)])
    with pytest.raises(wl.WilsonError):
        engine.rows_product([good, bad])
    with pytest.raises(ValueError):
        engine.rows_product([good, _rows([7, 13], [(1, 2), (3, 4)])])
    assert engine.rows_product([good[:0]]).size == 0


def _sharded(engine, lo, hi, world):
    b = colshard.column_pieces(lo, hi, world)
    parts = [colshard.search_piece(engine, lo, hi, b, r) for r in range(world)]
    held = [x for x in parts if x is not None]
    return b, engine.rows_product(held), colshard.finish_pieces(engine, lo, hi, b, parts)


@pytest.mark.parametrize("lo,hi,world", [(200, 564, 3), (2**31 - 1000, 2**31 + 1000, 2),
                                         (10**9, 10**9 + 20000, 8), (10**6, 10**6 + 5000, 1)])
def test_sharded_matches_one_call(engine, lo, hi, world):
    want = engine.search(lo, hi)
    b, prod, got = _sharded(engine, lo, hi, world)
    assert got.checksum == want.checksum and got.results == want.results
    rows, _ = engine.rows(lo, hi, q_cap=b[-1])      # the product over all columns in one call
    assert np.array_equal(prod["p"], rows["p"])
    assert np.array_equal(prod["s0"], rows["s0"]) and np.array_equal(prod["s1"], rows["s1"])
    # the pieces as gathered between ranks: 16-byte digit arrays plus the primes
    parts = [colshard.search_piece(engine, lo, hi, b, r) for r in range(world)]
    digs = [colshard.piece_digits(x) for x in parts if x is not None]
    prod2 = engine.rows_product(digs, p=rows["p"])
    assert np.array_equal(prod2["s0"], rows["s0"]) and np.array_equal(prod2["s1"], rows["s1"])


def test_sharded_case5_golden(engine, golden):
    k = golden["kat"][4]
    _, _, got = _sharded(engine, k["pmin"], k["pmax"], 4)
    assert "%016X" % got.checksum == k["checksum"] and len(got.results) == k["results"]


def test_sharded_case1_above_2_32(engine, golden):
    k = golden["kat"][0]
    b, _, got = _sharded(engine, k["pmin"], k["pmax"], 3)
    assert b[1] > 1 << 32
    assert "%016X" % got.checksum == k["checksum"]
    assert got.results == [(k["last_prime"], k["last_value"])]
