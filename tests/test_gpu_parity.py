"""CUDA engine vs the oracle and the golden vectors, through the C ABI.

Integer results must be bit-exact: T_p! mod p^2 digits, the quotient and
remainder of ((p-1)! + 1) mod p^2, result lines and checksums.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _oracle_built():
    oracle.build()


def _same_rows(got, want, fields=("p", "s0", "s1", "rem", "quot", "type")):
    assert len(got) == len(want)
    for f in fields:
        bad = np.nonzero(got[f].astype(np.uint64) != want[f].astype(np.uint64))[0]
        assert bad.size == 0, (f, [(int(got["p"][i]), int(got[f][i]), int(want[f][i])) for i in bad[:5]])


def test_small_golden(engine, golden):
    rows, st = engine.rows(5, 3000)
    want = {g["p"]: g for g in golden["small"]}
    assert len(rows) == len(want)
    for r in rows:
        g = want[int(r["p"])]
        assert (int(r["rem"]), int(r["quot"])) == (g["rem"], g["quot"]), int(r["p"])
        assert (int(r["s0"]), int(r["s1"])) == (g["tfact_s0"], g["tfact_s1"]), int(r["p"])
        assert int(r["status"]) == 0


def test_single_prime_ranges(engine, golden):
    # one prime per range: the class target is the prime's own target, no tail
    for g in golden["small"][::7]:
        rows, _ = engine.rows(g["p"], g["p"] + 1)
        assert (int(rows[0]["rem"]), int(rows[0]["quot"])) == (g["rem"], g["quot"])


def test_range_1e5(engine, golden):
    g = golden["range_1e5"]
    res = engine.search(g["pmin"], g["pmax"])
    assert res.lines() == g["lines"]
    assert "%016X" % res.checksum == g["checksum"]


def test_kat5(engine, golden):
    k = golden["kat"][4]
    res = engine.search(k["pmin"], k["pmax"])
    assert len(res.results) == k["results"]
    assert "%016X" % res.checksum == k["checksum"]
    assert res.results[-1] == (k["last_prime"], k["last_value"])
    assert res.stats.pi_maxtarget == k["pi_maxtarget"]


def test_kat6(engine, golden):
    k = golden["kat"][5]
    res = engine.search(k["pmin"], k["pmax"])
    assert "%016X" % res.checksum == k["checksum"]
    assert res.results == [(k["last_prime"], k["last_value"])]
    assert res.stats.pi_maxtarget == k["pi_maxtarget"]


@pytest.mark.parametrize("lo,hi", [
    (10**6, 10**6 + 30000),                 # 2 limbs
    (2**31 - 3000, 2**31 + 3000),           # straddles 2^31: 3 limbs for the whole range
    (3 * 10**9, 3 * 10**9 + 600),           # 3 limbs, class-2 target above 2^30
])
def test_full_parity_with_oracle(engine, lo, hi):
    got, _ = engine.rows(lo, hi)
    want, _ = oracle.search(lo, hi)
    _same_rows(got, want)
    assert np.all(got["status"] == 0)


def test_wide_columns_wilson_check(engine):
    # class-2 target above 2^31: columns q >= 2^31 take the conditional
    # subtraction; Wilson's theorem (rem == 0) checks every row
    lo = 4294967296 + 10**6
    rows, st = engine.rows(lo, lo + 3000)
    assert st.targets[2] > 2**31
    assert len(rows) > 50
    assert np.all(rows["status"] == 0) and np.all(rows["rem"] == 0)


def test_wide_columns_oracle_rows(engine):
    lo = 4294967296 + 10**6
    got, _ = engine.rows(lo, lo + 300)
    want, _ = oracle.search(lo, lo + 300)
    _same_rows(got, want)


@pytest.mark.parametrize("lo,hi,qcap", [
    (10**13, 10**13 + 10**7, 1 << 16),
    ((1 << 62) - 1 - 10**7, (1 << 62) - 1, 1 << 16),
    (4294967296 - 30000, 4294967296 + 30000, 1 << 16),
])
def test_capped_golden(engine, golden, lo, hi, qcap):
    case = next(c for c in golden["capped"] if c["pmin"] == lo)
    rows, st = engine.rows(lo, hi, q_cap=qcap)
    byp = {int(p): i for i, p in enumerate(rows["p"])}
    for w in case["rows"]:
        r = rows[byp[w["p"]]]
        assert (int(r["s0"]), int(r["s1"])) == (w["s0"], w["s1"]), w["p"]
    for t, T in case["targets"].items():
        assert st.targets[int(t)] == T


@pytest.mark.parametrize("lo,hi", [(10**13, 10**13 + 20000), ((1 << 62) - 1 - 20000, (1 << 62) - 1),
                                   ((1 << 47) - 2000, (1 << 47) + 2000)])   # 3 -> 4 limbs across the range
def test_capped_parity_with_oracle(engine, lo, hi):
    qcap = 1 << 20
    got, _ = engine.rows(lo, hi, q_cap=qcap)
    sel = list(range(0, len(got), max(1, len(got) // 24)))
    want, _ = oracle.search(lo, hi, qcap=qcap, rows=sel)
    for i in sel:
        assert (int(got["s0"][i]), int(got["s1"][i])) == (int(want["s0"][i]), int(want["s1"][i])), int(got["p"][i])


@pytest.mark.parametrize("lo,hi", [((1 << 62) - 1 - 60000, (1 << 62) - 1), (10**13, 10**13 + 60000)])
def test_dense_partial_tiles_with_oracle(engine, lo, hi):
    # Below 2^16 every column of these ranges is in the dense regime.  Their
    # class buckets hold 256 to 1,000 rows: full 256-row tiles, then a last
    # tile narrower than 256 lanes that runs one split per CTA, with the chunk
    # length of the full tiles.  Every row against the oracle.
    qcap = 1 << 16
    got, _ = engine.rows(lo, hi, q_cap=qcap)
    counts = [int((got["type"] == t).sum()) for t in range(3)]
    assert all(c > 256 and c % 256 for c in counts), counts
    want, _ = oracle.search(lo, hi, qcap=qcap)
    _same_rows(got, want, fields=("p", "s0", "s1", "type"))


def test_batch_matches_plain(engine):
    ranges = [(10**6, 10**6 + 5000), (10**8, 10**8 + 3000), (200, 564), (2**31 - 1000, 2**31 + 1000)]
    per, results, st = engine.batch(ranges)
    # the batch's sweep, merges, tail and lift ran as one CUDA graph (every
    # class target is below 2^32); the per-range calls launch them one by one
    assert st.graph_nodes > 0 and st.ms_sweep > 0
    for (lo, hi), pr in zip(ranges, per):
        one = engine.search(lo, hi)
        assert one.stats.graph_nodes == 0
        assert pr["checksum"] == one.checksum
        assert pr["results"] == len(one.results)
    # capped
    ranges = [(10**13, 10**13 + 10000), (10**9, 10**9 + 10000), ((1 << 62) - 30000, (1 << 62) - 1)]
    per, _, st = engine.batch(ranges, q_cap=1 << 22)
    assert st.graph_nodes > 0 and st.ms_sweep > 0
    for (lo, hi), pr in zip(ranges, per):
        rows, _ = engine.rows(lo, hi, q_cap=1 << 22)
        ck = int((rows["p"].astype(object) + rows["s0"].astype(object) + rows["s1"].astype(object)).sum()) % (1 << 64)
        assert pr["checksum"] == ck


def test_cfg1_wilson_check_and_sample(engine):
    # every prime in [1e9, 1e9+1e6): the full search, Wilson's theorem on every
    # row, and a sample of rows against the oracle
    lo, hi = 10**9, 10**9 + 10**6
    rows, st = engine.rows(lo, hi)
    assert len(rows) == st.tested > 48000
    assert np.all(rows["status"] == 0)
    sel = list(range(0, len(rows), len(rows) // 6)) + [len(rows) - 1]
    want, _ = oracle.search(lo, hi, rows=sel)
    for i in sel:
        for f in ("s0", "s1", "rem", "quot"):
            assert int(rows[f][i]) == int(want[f][i]), (f, int(rows["p"][i]))


def test_errors(engine):
    import clwilson_b200 as wl
    with pytest.raises(wl.WilsonError) as e:
        engine.search(4, 100)
    assert e.value.code == -1
    with pytest.raises(wl.WilsonError) as e:
        engine.search(24, 29)            # no primes in [24, 29)
    assert e.value.code == -3


def _range_oracle(args):
    p, T, lo, hi = args
    return oracle.range_product(p, T, lo, hi)


@pytest.mark.parametrize("lo,hi,nsample", [(10**13, 10**13 + 20000, 8), ((1 << 62) - 20001, (1 << 62) - 1, 4)])
def test_big_columns_against_oracle(engine, lo, hi, nsample):
    # capped(2^32 + 2^26) = capped(2^32) * prod_{2^32 <= q < 2^32 + 2^26} q^{v_q(T!)}:
    # the window sieve, the 64-bit sweep and the merge against the oracle
    from concurrent.futures import ThreadPoolExecutor
    q1, q2 = 1 << 32, (1 << 32) + (1 << 26)
    r1, st = engine.rows(lo, hi, q_cap=q1)
    r2, _ = engine.rows(lo, hi, q_cap=q2)
    idx = list(range(0, len(r1), max(1, len(r1) // nsample)))[:nsample]
    jobs = [(int(r1["p"][i]), st.targets[int(r1["type"][i])], q1, q2) for i in idx]
    with ThreadPoolExecutor(max_workers=8) as ex:
        parts = list(ex.map(_range_oracle, jobs))
    for i, (s0, s1) in zip(idx, parts):
        p = int(r1["p"][i])
        m = p * p
        a = int(r1["s0"][i]) + p * int(r1["s1"][i])
        b = int(r2["s0"][i]) + p * int(r2["s1"][i])
        assert a * (s0 + p * s1) % m == b, p


def test_kat1_columns_above_2_32(engine, golden):
    # self-test case 1: class target 2.07e11, columns up to it (cl_wilson.cpp:2007-2013)
    k = golden["kat"][0]
    res = engine.search(k["pmin"], k["pmax"])
    assert res.stats.pi_maxtarget == k["pi_maxtarget"]
    assert "%016X" % res.checksum == k["checksum"]
    assert res.results == [(k["last_prime"], k["last_value"])]


def test_large_least_cubic_nonresidue(engine, golden):
    # type-0 primes whose least cubic non-residue is 37 or 41 (the largest
    # below 1e8): the lift's search for c and u (k_finish, find.cl:71-117)
    # runs that far; exact (p-1)! + 1 mod p^2 from Python integers, and the
    # oracle's rows; then all of them as ranges of one batch
    ranges = []
    for g in golden["nonresidue"]:
        p = g["p"]
        rows, _ = engine.rows(p, p + 1)
        assert len(rows) == 1 and int(rows["status"][0]) == 0
        assert (int(rows["rem"][0]), int(rows["quot"][0])) == (g["rem"], g["quot"]), p
        want, _ = oracle.search(p, p + 1)
        assert (int(rows["s0"][0]), int(rows["s1"][0])) == (int(want["s0"][0]), int(want["s1"][0])), p
        ranges.append((p, p + 1))
    per, _, _ = engine.batch(ranges)
    for (p, _), pr, g in zip(ranges, per, golden["nonresidue"]):
        assert pr["checksum"] == (p + g["rem"] + g["quot"]) % (1 << 64) and pr["status"] == 0
