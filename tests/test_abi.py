"""The C ABI library: loads, exports every declared symbol, host-side logic (no GPU)."""
import ctypes
import os
import re

import pytest

import clwilson_b200 as wl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    import glob
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        names |= set(re.findall(r"\b(wl_[a-z0-9_]+)\s*\(", open(h).read()))
    return sorted(names)


def test_library_loads_and_exports_header_symbols():
    L = wl.load_library()
    syms = declared_symbols()
    assert syms, "no declarations found"
    for s in syms:
        assert hasattr(L, s), s
    assert set(wl.SYMBOLS) >= set(syms)


def test_bindings_match_header_arity():
    # every declared function has a ctypes binding with as many parameters as
    # its declaration (a mismatch passes garbage across the C ABI)
    import glob
    src = "".join(open(h).read() for h in glob.glob(os.path.join(ROOT, "include", "*.h")))
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    decls = re.findall(r"\b(?:int|void|const char\s*\*|void\s*\*)\s*\*?\s*(wl_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src)
    assert len(decls) >= len(declared_symbols())
    L = wl.load_library()
    for name, params in decls:
        p = params.strip()
        n = 0 if p in ("", "void") else p.count(",") + 1
        argtypes = getattr(L, name).argtypes
        assert argtypes is not None and len(argtypes) == n, (name, n, argtypes)


def test_strerror():
    L = wl.load_library()
    assert L.wl_strerror(-3) == b"there are no primes to test in this range!"
    assert L.wl_strerror(0) == b"ok"


def _ref_parse(s, lo, hi):
    """Python restatement of parse_uint64 (putil.c:34-116) for cross-checking."""
    import re as _re
    m = _re.match(r"^\s*([+-]?)(0[xX][0-9a-fA-F]+|0[0-7]*|[1-9][0-9]*)", s)
    if not m:
        num, tail = 0, s
    else:
        tok = m.group(2)
        num = int(tok, 16) if tok[:2].lower() == "0x" else (int(tok, 8) if tok.startswith("0") else int(tok))
        if m.group(1) == "-":
            num = (-num) % (1 << 64)
        tail = s[m.end():]
    if num > hi:
        return -2, 0
    c = tail[:1]
    if c in ("P", "T", "G", "M", "K"):
        if len(tail) != 1:
            return -1, 0
        for _ in range("KMGTP".index(c) + 1):
            if num > hi // 1000:
                return -2, 0
            num *= 1000
    elif c in ("e", "E"):
        rest = tail[1:]
        if rest and not rest.isdigit():
            return -1, 0
        for _ in range(int(rest or 0)):
            if num > hi // 10:
                return -2, 0
            num *= 10
    elif c in ("k", "m", "g", "t", "p"):
        if len(tail) != 1:
            return -1, 0
        e = 10 * ("kmgtp".index(c) + 1)
        if num > (hi >> e):
            return -2, 0
        num <<= e
    elif c in ("b", "B"):
        rest = tail[1:]
        if rest and not rest.isdigit():
            return -1, 0
        for _ in range(int(rest or 0)):
            if num > (hi >> 1):
                return -2, 0
            num <<= 1
    elif c != "":
        return -1, 0
    if num < lo:
        return -2, 0
    return 0, num


@pytest.mark.parametrize("text", ["5", "1000", "1e9", "1E3", "2K", "3M", "1G", "2T", "1P", "4k", "1m", "3g",
                                  "1b10", "0x10", "010", "12x", "1e", "5KK", "4611686018427387903",
                                  "4611686018427387904", "99999999999999999999", "4", "1p", "abc", "",
                                  "0K", "7b0", "9e0", "5e18", "1b62", "3p", "0x1Fe3", "5Q", "12e1x", "6b"])
def test_parse_uint64(text):
    lo, hi = 5, wl.WL_MAXP
    rc, v = wl.parse_uint64(text, lo, hi)
    want = _ref_parse(text, lo, hi)
    assert rc == want[0], text
    if rc == 0:
        assert v == want[1]


def test_range_rules():
    # setupSearch (cl_wilson.cpp:1146-1181) and the -p/-P bounds (main.cpp:50-56)
    assert wl.check_range(5, 6) == 0
    assert wl.check_range(4, 6) == -1
    assert wl.check_range(10, 10) == -1
    assert wl.check_range(10**9, 10**9 + 10**7) == 0
    assert wl.check_range(10**9, 10**9 + 10**7 + 1) == -1
    assert wl.check_range(wl.WL_MAXP - 10, wl.WL_MAXP) == 0
    assert wl.check_range(wl.WL_MAXP - 10, wl.WL_MAXP + 1) == -1


def test_results_file_format(tmp_path):
    path = str(tmp_path / "results.txt")
    wl.write_results(path, [(563, 0), (100519, 519), (87467099, -2)], 0x80A3)
    assert open(path).read() == ("563 is a Wilson prime\n100519 is a Near-Wilson prime +519\n"
                                 "87467099 is a Near-Wilson prime -2\n00000000000080A3\n")
    wl.write_results(path, [], 0x1234)
    assert open(path).read() == "no results\n0000000000001234\n"
