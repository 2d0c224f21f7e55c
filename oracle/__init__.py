"""CPU oracle for the Wilson-prime search (test infrastructure only).

Python bindings for ``wilson_oracle.c``, a C restatement of mfl0p/CLWilson's
search algorithm (kernels/common.cl, setup.cl, mulsmall.cl, iterate.cl,
find.cl; cl_wilson.cpp:691-900, 1293-1365, 1549-1586).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its CPU baseline
legs) may import this package: it is the checker and the timed CPU baseline,
never part of the engine.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "wilson_oracle.c")
LIB = os.path.join(HERE, "liboracle.so")


class OrcRow(ctypes.Structure):
    _fields_ = [
        ("p", ctypes.c_uint64),
        ("s0", ctypes.c_uint64),
        ("s1", ctypes.c_uint64),
        ("rem", ctypes.c_uint64),
        ("quot", ctypes.c_uint64),
        ("type", ctypes.c_uint32),
        ("status", ctypes.c_int32),
    ]


ROW_DTYPE = np.dtype(
    [("p", "<u8"), ("s0", "<u8"), ("s1", "<u8"), ("rem", "<u8"), ("quot", "<u8"),
     ("type", "<u4"), ("status", "<i4")]
)


def build(force: bool = False) -> str:
    """Compile the oracle with gcc (-O3, OpenMP) into oracle/liboracle.so."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-fopenmp", "-shared", "-fPIC", "-std=c11",
           "-Wall", "-Wno-unused-function", SRC, "-o", LIB + ".tmp"]
    subprocess.check_call(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        u64, u32, i64p = ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(ctypes.c_int64)
        L.orc_search.restype = ctypes.c_long
        L.orc_search.argtypes = [u64, u64, u64, ctypes.c_int, ctypes.POINTER(u32), ctypes.c_size_t,
                                 ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(u64)]
        L.orc_list_primes.restype = ctypes.c_size_t
        L.orc_list_primes.argtypes = [u64, u64, ctypes.c_void_p, ctypes.c_size_t]
        L.orc_is_prime.restype = ctypes.c_int
        L.orc_is_prime.argtypes = [u64]
        L.orc_isqrt.restype = u64
        L.orc_isqrt.argtypes = [u64]
        for fn in ("orc_find_a_brute", "orc_find_c_brute", "orc_find_u_brute", "orc_cornacchia_a"):
            getattr(L, fn).restype = ctypes.c_int
            getattr(L, fn).argtypes = [u64, i64p]
        L.orc_cornacchia_cu.restype = ctypes.c_int
        L.orc_cornacchia_cu.argtypes = [u64, i64p, i64p]
        L.orc_factorial_mod_p2.restype = None
        L.orc_factorial_mod_p2.argtypes = [u64, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.orc_small_factorial.restype = None
        L.orc_small_factorial.argtypes = [u64, u64, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.orc_lift_digits.restype = ctypes.c_int
        L.orc_lift_digits.argtypes = [u64, u64, u64, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        L.orc_count_primes_below.restype = ctypes.c_size_t
        L.orc_count_primes_below.argtypes = [u64]
        L.orc_threads.restype = ctypes.c_int
        L.orc_range_product.restype = None
        L.orc_range_product.argtypes = [u64, u64, u64, u64, ctypes.POINTER(u64), ctypes.POINTER(u64)]
        _lib = L
    return _lib


def search(pmin: int, pmax: int, qcap: int = 0, threads: int = 0, rows=None):
    """Rows (numpy structured array) and class targets for all primes in [pmin, pmax).

    qcap == 0 is the full search; qcap > 0 the capped partial product over
    sieving primes q < qcap.  ``rows`` selects a subset of row indices.
    """
    L = lib()
    n = L.orc_list_primes(pmin, pmax, None, 0)
    out = np.zeros(n, dtype=ROW_DTYPE)
    tg = (ctypes.c_uint64 * 3)()
    sel_p, nsel = None, 0
    if rows is not None:
        sel = np.ascontiguousarray(np.asarray(rows, dtype=np.uint32))
        sel_p, nsel = sel.ctypes.data_as(ctypes.POINTER(ctypes.c_uint32)), sel.size
    got = L.orc_search(pmin, pmax, qcap, threads, sel_p, nsel, out.ctypes.data, n, tg)
    if got < 0:
        raise RuntimeError("oracle search failed")
    return out, [int(x) for x in tg]


def list_primes(lo: int, hi: int) -> np.ndarray:
    L = lib()
    n = L.orc_list_primes(lo, hi, None, 0)
    out = np.zeros(n, dtype=np.uint64)
    L.orc_list_primes(lo, hi, out.ctypes.data, n)
    return out


def _i64_call(fn, *args):
    r = ctypes.c_int64()
    rc = fn(*args, ctypes.byref(r))
    return None if rc else r.value


def find_a_brute(p): return _i64_call(lib().orc_find_a_brute, p)
def find_c_brute(p): return _i64_call(lib().orc_find_c_brute, p)
def find_u_brute(p): return _i64_call(lib().orc_find_u_brute, p)
def cornacchia_a(p): return _i64_call(lib().orc_cornacchia_a, p)


def cornacchia_cu(p):
    c, u = ctypes.c_int64(), ctypes.c_int64()
    rc = lib().orc_cornacchia_cu(p, ctypes.byref(c), ctypes.byref(u))
    return None if rc else (c.value, u.value)


def factorial_mod_p2(p: int):
    s0, s1 = ctypes.c_uint64(), ctypes.c_uint64()
    lib().orc_factorial_mod_p2(p, ctypes.byref(s0), ctypes.byref(s1))
    return s0.value, s1.value


def small_factorial(p: int, T: int):
    s0, s1 = ctypes.c_uint64(), ctypes.c_uint64()
    lib().orc_small_factorial(p, T, ctypes.byref(s0), ctypes.byref(s1))
    return s0.value, s1.value


def range_product(p: int, T: int, qlo: int, qhi: int):
    """Digits of prod_{qlo <= q < qhi, q prime} q^{v_q(T!)} mod p^2."""
    s0, s1 = ctypes.c_uint64(), ctypes.c_uint64()
    lib().orc_range_product(p, T, qlo, qhi, ctypes.byref(s0), ctypes.byref(s1))
    return s0.value, s1.value


def lift_digits(p: int, s0: int, s1: int):
    rem, quot = ctypes.c_uint64(), ctypes.c_uint64()
    rc = lib().orc_lift_digits(p, s0, s1, ctypes.byref(rem), ctypes.byref(quot))
    return None if rc else (rem.value, quot.value)


def is_prime(n: int) -> bool:
    return bool(lib().orc_is_prime(n))


def count_primes_below(n: int) -> int:
    return int(lib().orc_count_primes_below(n))


def checksum(rows) -> int:
    """Sum of p + rem + quot mod 2^64 (cl_wilson.cpp:900)."""
    s = (rows["p"].astype(object) + rows["rem"].astype(object) + rows["quot"].astype(object)).sum()
    return int(s) & ((1 << 64) - 1)


def partial_checksum(rows) -> int:
    """Sum of p + s0 + s1 mod 2^64 over rows (capped-sweep checksum)."""
    s = (rows["p"].astype(object) + rows["s0"].astype(object) + rows["s1"].astype(object)).sum()
    return int(s) & ((1 << 64) - 1)


def result_lines(rows):
    """results.txt lines in ascending p (cl_wilson.cpp:657-688, 872-898)."""
    lines = []
    for r in rows:
        p, quot = int(r["p"]), int(r["quot"])
        neg = p - quot
        smallest = min(quot, neg)
        if quot == 0:
            lines.append(f"{p} is a Wilson prime")
        elif smallest < 1000:
            dq = quot if smallest == quot else -neg
            lines.append(f"{p} is a Near-Wilson prime {dq:+d}")
    return lines
