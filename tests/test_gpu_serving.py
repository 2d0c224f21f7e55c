"""Serving sessions (wl_server_*): continuous batching over a resident row pool.

Each request's rows, result lines and checksum must be bit-identical to the
one-shot engine (wl_search / wl_rows) on the same range, whether the request
runs alone or shares the GPU's column sweeps with other requests, whatever
the step size (column chunking) and however full the row pool is (queueing).
"""
import numpy as np
import pytest

import clwilson_b200 as wl

pytestmark = pytest.mark.gpu

FULL = [(200, 564), (10**6, 10**6 + 5000), (2**31 - 1000, 2**31 + 1000), (10**9, 10**9 + 20000)]
CAPPED = [(10**13, 10**13 + 10000, 1 << 22), ((1 << 62) - 30000, (1 << 62) - 1, 1 << 22),
          (10**9, 10**9 + 10000, 1 << 22), (10**8, 10**8 + 4000, 1 << 20)]


@pytest.fixture(scope="module")
def expected(engine):
    exp = {}
    for lo, hi in FULL:
        r = engine.search(lo, hi)
        rows, _ = engine.rows(lo, hi)
        exp[(lo, hi, 0)] = (r.checksum, r.results, rows)
    for lo, hi, q in CAPPED:
        rows, _ = engine.rows(lo, hi, q_cap=q)
        ck = int((rows["p"].astype(object) + rows["s0"].astype(object) + rows["s1"].astype(object)).sum()) % (1 << 64)
        exp[(lo, hi, q)] = (ck, [], rows)
    return exp


def _check(srv, rid, key, expected):
    info = srv.wait(rid, 600_000)
    assert info.state == "done", (key, info)
    ck, results, rows = expected[key]
    assert info.checksum == ck, key
    assert info.tested == len(rows)
    got = srv.rows(rid)
    for f in ("p", "s0", "s1", "rem", "quot", "type"):
        assert np.array_equal(got[f], rows[f]), (key, f)
    if key[2] == 0:
        assert srv.results(rid) == results
    return info


def _all_keys():
    return [(lo, hi, 0) for lo, hi in FULL] + list(CAPPED)


def test_alone(expected):
    with wl.Server(0) as srv:
        for key in _all_keys():
            rid = srv.submit(*key)
            _check(srv, rid, key, expected)
            srv.release(rid)


@pytest.mark.parametrize("step_cells,shares", [(0, "least-work"), (1 << 24, "least-work"), (1 << 24, "equal")])
def test_mixed(expected, step_cells, shares):
    # everything at once, and a second wave submitted while the first runs
    with wl.Server(0, step_cells=step_cells, shares=shares) as srv:
        keys = _all_keys()
        ids = [srv.submit(*k) for k in keys]
        ids2 = [srv.submit(*k) for k in reversed(keys)]
        for rid, k in zip(ids + ids2, keys + list(reversed(keys))):
            _check(srv, rid, k, expected)
        st = srv.stats()
        assert st["completed"] == 2 * len(keys) and st["failed"] == 0
        assert st["peak_active"] > 1


def test_small_pool_queues(expected):
    # a pool of 2500 rows: the 1e9 full range (~980 rows) and the capped ones
    # (~300-1500 rows) cannot all be resident; they queue and still match
    with wl.Server(0, pool_bytes=2500 * wl.SERVER_ROW_BYTES, step_cells=1 << 26) as srv:
        keys = _all_keys()
        ids = [srv.submit(*k) for k in keys]
        infos = [_check(srv, rid, k, expected) for rid, k in zip(ids, keys)]
        assert srv.stats()["peak_rows"] <= 2500
        assert max(i.ms_queued for i in infos) > 0


def test_cancel_and_errors(expected):
    with wl.Server(0, step_cells=1 << 24) as srv:
        big = srv.submit(10**13, 10**13 + 10**6, 1 << 30)     # long-running
        small = srv.submit(*CAPPED[0])
        srv.cancel(big)
        assert srv.wait(big, 600_000).state == "cancelled"
        _check(srv, small, CAPPED[0], expected)
        # no primes in [24, 29)
        none = srv.submit(24, 29)
        info = srv.wait(none, 600_000)
        assert info.state == "failed" and info.rc == -3
        with pytest.raises(wl.WilsonError):
            srv.submit(4, 100)
        # the server keeps serving after failures
        rid = srv.submit(*CAPPED[3])
        _check(srv, rid, CAPPED[3], expected)


def test_columns_above_2_32(engine, golden):
    # self-test cases 1 and 2 (class targets 2.07e11 and 2.77e11, cl_wilson.cpp:2007-2030):
    # their columns above 2^32 are sieved in chunks inside the step loop.  Alone,
    # then together with small requests that keep arriving; and a capped request
    # whose cap lies above 2^32.
    kats = golden["kat"][:2]
    small = [(lo, hi, 0) for lo, hi in FULL[:2]] + [CAPPED[2], CAPPED[3]]
    want_small = {}
    for lo, hi, q in small:
        rows, _ = engine.rows(lo, hi, q_cap=q)
        want_small[(lo, hi, q)] = rows
    cap = (1 << 32) + (1 << 26)
    capped_rows, _ = engine.rows(10**13, 10**13 + 2000, q_cap=cap)

    def check_kat(srv, rid, k):
        info = srv.wait(rid, 600_000)
        assert info.state == "done", info
        assert "%016X" % info.checksum == k["checksum"]
        assert srv.results(rid) == [(k["last_prime"], k["last_value"])]

    def check_small(srv, rid, key):
        info = srv.wait(rid, 600_000)
        assert info.state == "done", (key, info)
        got = srv.rows(rid)
        for f in ("p", "s0", "s1", "rem", "quot"):
            assert np.array_equal(got[f], want_small[key][f]), (key, f)
        return info.ms_latency

    with wl.Server(0) as srv:
        for k in kats:
            check_kat(srv, srv.submit(k["pmin"], k["pmax"]), k)
        rid = srv.submit(10**13, 10**13 + 2000, cap)
        assert srv.wait(rid, 600_000).state == "done"
        got = srv.rows(rid)
        assert np.array_equal(got["s0"], capped_rows["s0"]) and np.array_equal(got["s1"], capped_rows["s1"])
        alone = [check_small(srv, srv.submit(*key), key) for key in small]
        # mixed: both long requests, then small ones submitted while they run
        big = [srv.submit(k["pmin"], k["pmax"]) for k in kats]
        mixed = []
        for _ in range(3):
            ids = [(srv.submit(*key), key) for key in small]
            mixed += [check_small(srv, rid, key) for rid, key in ids]
        for rid, k in zip(big, kats):
            check_kat(srv, rid, k)
        st = srv.stats()
        assert st["failed"] == 0 and st["peak_active"] > 1
    assert len(alone) == len(small) and len(mixed) == 3 * len(small)


@pytest.mark.parametrize("lo,hi,q", [(10**6, 10**6 + 5000, 0), (10**13, 10**13 + 4000, 1 << 20),
                                     ((1 << 62) - 8000, (1 << 62) - 1, 1 << 20)])
def test_one_request_per_limb_width_against_oracle(lo, hi, q):
    # 2-, 3- and 4-limb rows served alone, checked against the oracle directly
    import oracle
    with wl.Server(0) as srv:
        rid = srv.submit(lo, hi, q)
        info = srv.wait(rid, 600_000)
        assert info.state == "done", info
        got = srv.rows(rid)
    sel = list(range(0, len(got), max(1, len(got) // 16)))
    want, _ = oracle.search(lo, hi, qcap=q, rows=sel)
    assert np.array_equal(got["p"], want["p"])
    fields = ("s0", "s1") if q else ("s0", "s1", "rem", "quot")
    for i in sel:
        for f in fields:
            assert int(got[f][i]) == int(want[f][i]), (lo, f, int(got["p"][i]))
