"""Generate the golden vectors under tests/golden/ with exact Python integers.

Nothing here uses the oracle or the engine: every value is computed from its
mathematical definition (Python big integers), or transcribed from the
reference's built-in self-test, so the fixtures pin both independently.

  kat.json         the reference's seven self-test cases (cl_wilson.cpp:2007-2115)
  small.json       every prime 5 <= p < 3000: (p-1)! + 1 mod p^2 as (rem, quot),
                   the class, and T_p! mod p^2 digits (T_p = (p-1)/6, /4, /2)
  range_1e5.json   the full search of [100000, 101000): result lines, checksum
  capped.json      capped partial products prod_{q < Q, q <= T} q^{v_q(T!)} mod p^2
                   for test primes of the mid-size and top-of-range workloads
  nonresidue.json  the primes p = 1 mod 3 below 1e8 whose least cubic non-residue
                   is 37 or more (the lift's c and u come from a search for one),
                   with (p-1)! + 1 mod p^2 as (rem, quot)

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def is_prime(n: int) -> bool:
    if n < 2:
        return False
    small = [2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37]
    for p in small:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in small:
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def primes_below(n: int):
    sieve = bytearray([1]) * n
    sieve[0:2] = b"\x00\x00"
    for i in range(2, int(n ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = bytearray(len(sieve[i * i::i]))
    return [i for i in range(n) if sieve[i]]


def cls(p: int):
    if p % 3 == 1:
        return 0, (p - 1) // 6
    if p % 12 == 5:
        return 1, (p - 1) // 4
    return 2, (p - 1) // 2


def fact_mod(n: int, m: int) -> int:
    f = 1
    for k in range(2, n + 1):
        f = f * k % m
    return f


def legendre(q: int, T: int) -> int:
    e, qq = 0, q
    while qq <= T:
        e += T // qq
        qq *= q
    return e


def result_line(p: int, quot: int):
    neg = p - quot
    smallest = min(quot, neg)
    if quot == 0:
        return f"{p} is a Wilson prime"
    if smallest < 1000:
        dq = quot if smallest == quot else -neg
        return f"{p} is a Near-Wilson prime {dq:+d}"
    return None


def kat():
    # cl_wilson.cpp:2007-2115: (pmin, pmax, result count, checksum, pi(maxtarget),
    # last result prime, signed result)
    cases = [
        (1239053554603, 1239053554604, 1, 0x00000240FAB1A752, 8257082014, 1239053554603, -4, "2007-2013"),
        (1108967825921, 1108967825922, 1, 0x0000010233A2220D, 10956003002, 1108967825921, 12, "2024-2030"),
        (5609877309359, 5609877309360, 1, 0x00000A344D7D0F58, 101542897873, 5609877309359, -6, "2041-2047"),
        (16556218163369, 16556218163370, 1, 0x00000F0ECB80A0AB, 147755473426, 16556218163369, 2, "2058-2064"),
        (200, 564, 57, 0x00000000000080A3, 30, 563, 0, "2075-2081"),
        (86000000, 87467200, 1, 0x0000097C61AB0943, 2604536, 87467099, -2, "2092-2098"),
        (17524177394450, 17524177394618, 1, 0x00005B54B4CBBC47, 304620766446, 17524177394617, 256, "2109-2115"),
    ]
    out = []
    for i, (a, b, n, ck, pi, lp, lv, lines) in enumerate(cases, 1):
        out.append({"case": i, "pmin": a, "pmax": b, "results": n, "checksum": "%016X" % ck,
                    "pi_maxtarget": pi, "last_prime": lp, "last_value": lv,
                    "source": f"cl_wilson.cpp:{lines}"})
    return out


def small():
    rows = []
    for p in range(5, 3000):
        if not is_prime(p):
            continue
        m = p * p
        t, T = cls(p)
        v = (fact_mod(p - 1, m) + 1) % m
        tf = fact_mod(T, m)
        rows.append({"p": p, "type": t, "T": T, "rem": v % p, "quot": v // p,
                     "tfact_s0": tf % p, "tfact_s1": tf // p})
    return rows


def range_search(pmin: int, pmax: int):
    rows, lines, ck = [], [], 0
    for p in range(pmin, pmax):
        if not is_prime(p):
            continue
        m = p * p
        v = (fact_mod(p - 1, m) + 1) % m
        rem, quot = v % p, v // p
        ck = (ck + p + rem + quot) & ((1 << 64) - 1)
        rows.append({"p": p, "rem": rem, "quot": quot})
        ln = result_line(p, quot)
        if ln:
            lines.append(ln)
    return {"pmin": pmin, "pmax": pmax, "rows": rows, "lines": lines, "checksum": "%016X" % ck}


def capped(pmin: int, pmax: int, qcap: int, take: int):
    """First `take` test primes of [pmin, pmax): partial products over q < qcap
    with the Legendre exponents of the range's shared class targets."""
    tps = []
    p = pmin
    while p < pmax and len(tps) < 4 * take:
        if is_prime(p):
            tps.append(p)
        p += 1
    targets = {}
    for p in tps:
        t, T = cls(p)
        targets.setdefault(t, T)
    qs = primes_below(qcap)
    rows = []
    for p in tps[:take]:
        t, _ = cls(p)
        T = targets[t]
        m = p * p
        acc = 1
        for q in qs:
            if q > T:
                break
            acc = acc * pow(q, legendre(q, T), m) % m
        rows.append({"p": p, "type": t, "s0": acc % p, "s1": acc // p})
    return {"pmin": pmin, "pmax": pmax, "qcap": qcap, "targets": {str(k): v for k, v in targets.items()},
            "rows": rows}


def nonresidue(limit: int = 10 ** 8, least: int = 37):
    sieve = bytearray([1]) * limit
    sieve[0:2] = b"\x00\x00"
    for i in range(2, int(limit ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = bytearray(len(sieve[i * i::i]))
    gs = [g for g in range(2, 200) if sieve[g]]
    rows = []
    for p in range(7, limit, 6):          # p = 1 mod 6
        if not sieve[p]:
            continue
        e = (p - 1) // 3
        g = next(g for g in gs if pow(g, e, p) != 1)
        if g < least:
            continue
        m = p * p
        v = (fact_mod(p - 1, m) + 1) % m
        rows.append({"p": p, "type": 0, "least_cubic_nonresidue": g, "rem": v % p, "quot": v // p})
    return rows


def main():
    def dump(name, obj):
        with open(os.path.join(HERE, name), "w") as f:
            json.dump(obj, f, indent=1)
            f.write("\n")

    dump("kat.json", kat())
    dump("small.json", small())
    dump("range_1e5.json", range_search(100000, 101000))
    dump("capped.json", [
        capped(10 ** 13, 10 ** 13 + 10 ** 7, 1 << 16, 6),
        capped((1 << 62) - 1 - 10 ** 7, (1 << 62) - 1, 1 << 16, 6),
        capped(4294967296 - 30000, 4294967296 + 30000, 1 << 16, 6),
    ])
    dump("nonresidue.json", nonresidue())


if __name__ == "__main__":
    main()
