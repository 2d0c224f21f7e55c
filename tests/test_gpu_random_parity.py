"""Seeded random ranges over the whole input domain against the oracle.

Ranges from numpy default_rng(2024) have starts log-uniform in [5, 2^62 - 4000)
and widths log-uniform in [1, 3000], so they cover every limb width and the
boundaries between them:
* capped at a column bound drawn log-uniformly from [2^6, 2^22] per range
  (so the dense / prefix-fold split point falls anywhere): every row's
  digits (s0, s1), class and prime equal the oracle's; a range without
  primes fails with WL_ERR_NOPRIMES, as cl_wilson.cpp:1532-1536 stops;
* the same ranges in one wl_batch at q < 2^18: per-range checksums and counts
  equal the one-range calls';
* ranges below 1e7, searched in full: rows (rem, quot, status), result lines
  and checksum equal the oracle's.
"""
import numpy as np
import pytest

import clwilson_b200 as wl
import oracle

pytestmark = pytest.mark.gpu

QCAP = 1 << 18


def _ranges(seed, n, lo, hi, wmax):
    rng = np.random.default_rng(seed)
    starts = np.exp(rng.uniform(np.log(lo), np.log(hi), n))
    widths = np.exp(rng.uniform(0.0, np.log(wmax), n))
    out = []
    for s, w in zip(starts, widths):
        a = max(5, int(s))
        out.append((a, min(a + max(1, int(w)), (1 << 62) - 1)))
    return out


CAPPED = _ranges(2024, 96, 5.0, float((1 << 62) - 4000), 3000)
CAPS = [int(x) for x in np.exp(np.random.default_rng(2026).uniform(np.log(2.0**6), np.log(2.0**22), len(CAPPED)))]
FULL = _ranges(2025, 32, 5.0, 1e7, 3000)


@pytest.fixture(scope="module", autouse=True)
def _oracle_built():
    oracle.build()


def _rows_or_empty(engine, lo, hi, q_cap):
    try:
        return engine.rows(lo, hi, q_cap=q_cap)[0]
    except wl.WilsonError as e:
        assert e.code == -3, (lo, hi, e)     # WL_ERR_NOPRIMES
        return None


def test_random_capped_rows(engine):
    nonempty = 0
    for (lo, hi), cap in zip(CAPPED, CAPS):
        want, _ = oracle.search(lo, hi, qcap=cap)
        got = _rows_or_empty(engine, lo, hi, cap)
        if got is None:
            assert len(want) == 0, (lo, hi)
            continue
        nonempty += 1
        assert len(got) == len(want), (lo, hi)
        for f in ("p", "s0", "s1", "type"):
            bad = np.nonzero(got[f].astype(np.uint64) != want[f].astype(np.uint64))[0]
            assert bad.size == 0, (lo, hi, f, [int(got["p"][i]) for i in bad[:5]])
    assert nonempty >= 60


def test_random_batch_matches_one_range_calls(engine):
    ranges = [(lo, hi) for lo, hi in CAPPED if len(oracle.list_primes(lo, hi))]
    per, _, _ = engine.batch(ranges, q_cap=QCAP)
    for (lo, hi), pr in zip(ranges, per):
        rows, _ = engine.rows(lo, hi, q_cap=QCAP)
        assert pr["tested"] == len(rows)
        assert pr["checksum"] == oracle.partial_checksum(rows), (lo, hi)


def test_random_full_searches(engine):
    for lo, hi in FULL:
        want, _ = oracle.search(lo, hi)
        if len(want) == 0:
            with pytest.raises(wl.WilsonError):
                engine.search(lo, hi)
            continue
        got, _ = engine.rows(lo, hi)
        for f in ("p", "s0", "s1", "rem", "quot", "type", "status"):
            assert np.array_equal(got[f].astype(np.uint64), want[f].astype(np.uint64)), (lo, hi, f)
        res = engine.search(lo, hi)
        assert res.checksum == oracle.checksum(want), (lo, hi)
        assert [wl.result_line(p, v) for p, v in res.results] == oracle.result_lines(want), (lo, hi)
