"""The CPU oracle against the golden vectors (no GPU).

The oracle restates the reference's algorithm (oracle/wilson_oracle.c); these
tests pin it to values computed independently: exact Python integers
(tests/golden/make_golden.py) and the reference's self-test answers
(cl_wilson.cpp:2007-2115).
"""
import os

import numpy as np
import pytest

import oracle

SLOW = os.environ.get("CLW_SLOW") == "1"


@pytest.fixture(scope="module", autouse=True)
def _built():
    oracle.build()


def test_small_primes_against_exact_factorials(golden):
    # every prime 5 <= p < 3000, one range per prime so the class target is T_p itself
    for g in golden["small"]:
        p = g["p"]
        rows, tg = oracle.search(p, p + 1)
        assert len(rows) == 1
        r = rows[0]
        assert int(r["type"]) == g["type"]
        assert (int(r["rem"]), int(r["quot"])) == (g["rem"], g["quot"]), p
        assert (int(r["s0"]), int(r["s1"])) == (g["tfact_s0"], g["tfact_s1"]), p
        assert int(r["status"]) == 0


def test_one_range_against_exact_factorials(golden):
    # all primes < 3000 in one range: shared class targets plus the iterate tail
    rows, tg = oracle.search(5, 3000)
    want = {g["p"]: g for g in golden["small"]}
    assert len(rows) == len(want)
    for r in rows:
        g = want[int(r["p"])]
        assert (int(r["rem"]), int(r["quot"])) == (g["rem"], g["quot"])
        assert (int(r["s0"]), int(r["s1"])) == (g["tfact_s0"], g["tfact_s1"])


def test_range_1e5(golden):
    g = golden["range_1e5"]
    rows, _ = oracle.search(g["pmin"], g["pmax"])
    assert [int(x) for x in rows["p"]] == [r["p"] for r in g["rows"]]
    assert [int(x) for x in rows["quot"]] == [r["quot"] for r in g["rows"]]
    assert oracle.result_lines(rows) == g["lines"]
    assert "%016X" % oracle.checksum(rows) == g["checksum"]


def test_kat5_wilson_563(golden):
    k = golden["kat"][4]
    rows, tg = oracle.search(k["pmin"], k["pmax"])
    lines = oracle.result_lines(rows)
    assert len(lines) == k["results"] == 57
    assert "%016X" % oracle.checksum(rows) == k["checksum"]
    assert lines[-1] == "563 is a Wilson prime"
    assert oracle.count_primes_below(max(tg) + 1) == k["pi_maxtarget"]


@pytest.mark.skipif(not SLOW, reason="about two minutes on 8 cores; set CLW_SLOW=1")
def test_kat6_full(golden):
    k = golden["kat"][5]
    rows, tg = oracle.search(k["pmin"], k["pmax"])
    lines = oracle.result_lines(rows)
    assert "%016X" % oracle.checksum(rows) == k["checksum"]
    assert lines == [f"{k['last_prime']} is a Near-Wilson prime {k['last_value']:+d}"]


def test_kat6_targets(golden):
    # pi(maxtarget) of self-test case 6 (cl_wilson.cpp:2094)
    k = golden["kat"][5]
    ps = oracle.list_primes(k["pmin"], k["pmin"] + 200)
    first2 = next(int(p) for p in ps if p % 12 == 11)
    assert oracle.count_primes_below((first2 - 1) // 2 + 1) == k["pi_maxtarget"]


def test_wilson_primes():
    for p in (5, 13, 563):
        rows, _ = oracle.search(p, p + 1)
        assert int(rows[0]["quot"]) == 0 and int(rows[0]["rem"]) == 0


def test_capped_partials(golden):
    for case in golden["capped"]:
        rows, tg = oracle.search(case["pmin"], case["pmax"], qcap=case["qcap"],
                                 rows=list(range(len(case["rows"]))))
        for want in case["rows"]:
            r = rows[list(rows["p"]).index(want["p"])]
            assert int(r["status"]) == 1
            assert (int(r["s0"]), int(r["s1"])) == (want["s0"], want["s1"]), want["p"]
        for t, T in case["targets"].items():
            assert tg[int(t)] == T


def test_representations_against_reference_search():
    ps = [int(p) for p in oracle.list_primes(7, 60000)] + [int(p) for p in oracle.list_primes(10**12, 10**12 + 2000)]
    for p in ps:
        if p % 4 == 1:
            assert oracle.cornacchia_a(p) == oracle.find_a_brute(p), p
        if p % 3 == 1:
            c, u = oracle.cornacchia_cu(p)
            assert c == oracle.find_c_brute(p), p
            umod = 1 if ((p - 1) // 6) % 2 == 0 else 2
            assert (4 * p - u * u) % 3 == 0 and u % 3 == umod


def test_lift_independent_of_u():
    # every admissible u gives the same (p-1)! (cl_wilson.cpp:731-794 with any u from findu)
    for p in [int(x) for x in oracle.list_primes(7, 4000) if x % 3 == 1]:
        s0, s1 = oracle.small_factorial(p, (p - 1) // 6)
        got = oracle.lift_digits(p, s0, s1)
        m = p * p
        f = 1
        for k in range(2, p):
            f = f * k % m
        v = (f + 1) % m
        assert got == (v % p, v // p), p


def test_primality_against_sieve():
    lo, hi = 10**9, 10**9 + 200000
    got = oracle.list_primes(lo, hi)
    n = hi
    sieve = np.ones(n - lo, dtype=bool)
    for q in range(2, int(hi ** 0.5) + 1):
        start = max(q * q, (lo + q - 1) // q * q)
        sieve[start - lo::q] = False
    want = np.nonzero(sieve)[0] + lo
    assert np.array_equal(got, want.astype(np.uint64))


def test_large_least_cubic_nonresidue(golden):
    # primes whose least cubic non-residue is 37 or 41, the largest below 1e8:
    # the lift's search for c and u runs that far; (p-1)! + 1 mod p^2 from exact
    # integers, and Cornacchia's c equal to the reference's brute-force one
    # (find.cl:71-92); any u with 4p = u^2 + 3v^2 and the sign rule works
    assert len(golden["nonresidue"]) == 8
    for g in golden["nonresidue"]:
        p = g["p"]
        assert all(pow(k, (p - 1) // 3, p) == 1 for k in range(2, g["least_cubic_nonresidue"]))
        c, u = oracle.cornacchia_cu(p)
        assert c == oracle.find_c_brute(p)
        v2 = (4 * p - u * u) // 3
        assert 3 * v2 + u * u == 4 * p and int(round(v2 ** 0.5)) ** 2 == v2
        rows, _ = oracle.search(p, p + 1)
        assert (int(rows[0]["rem"]), int(rows[0]["quot"])) == (g["rem"], g["quot"]) and int(rows[0]["status"]) == 0
