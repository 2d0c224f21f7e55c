"""wl_column_product_noalloc: the column product without device allocation.

The entry point serves callers that own all device memory themselves and may
not allocate while they run; it keeps its intermediates in a fixed array
inside the library.  This test is the caller here: it allocates the inputs and
outputs with torch, calls the entry point through the C ABI twice in a row
(the second call reuses the scratch the first one left behind), and checks
each result bit for bit against the existing entry point wl_rows on the same
primes.  It sits in a file of its own that pytest collects last.
"""
import ctypes

import numpy as np
import pytest

import clwilson_b200 as wl

pytestmark = pytest.mark.gpu

QCAP = 1 << 20


def _primes_below(n):
    s = np.ones(n, dtype=bool)
    s[:2] = False
    for q in range(2, int(n ** 0.5) + 1):
        if s[q]:
            s[q * q::q] = False
    return np.nonzero(s)[0]


def _noalloc(L, primes, p_bound, T, cols):
    import torch
    dp = torch.tensor(primes.astype(np.int64), device="cuda")
    dc = torch.tensor(cols.astype(np.int32), device="cuda")
    out = torch.zeros(2 * len(primes), dtype=torch.int64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = L.wl_column_product_noalloc(dp.data_ptr(), len(primes), p_bound, T, dc.data_ptr(), len(cols),
                                     out.data_ptr(), stream)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy().astype(np.uint64).reshape(-1, 2)


@pytest.mark.parametrize("lo,hi,cls", [
    (10**9, 10**9 + 20000, 0),                       # 2-limb residues
    (10**13, 10**13 + 20000, 2),                     # 3-limb residues
])
def test_noalloc_matches_rows_twice(engine, lo, hi, cls):
    L = wl.load_library()
    rows, st = engine.rows(lo, hi, q_cap=QCAP)
    T = st.targets[cls]
    sel = rows[rows["type"] == cls]
    assert len(sel) > 100
    allq = _primes_below(QCAP)
    cols = allq[allq <= T]
    for call in range(2):
        rc, got = _noalloc(L, sel["p"], hi, T, cols)
        assert rc == 0, (call, L.wl_strerror(rc))
        assert np.array_equal(got[:, 0], sel["s0"]), call
        assert np.array_equal(got[:, 1], sel["s1"]), call


def test_noalloc_top_of_range_and_limits(engine):
    L = wl.load_library()
    hi = (1 << 62) - 1
    lo = hi - 20000
    rows, st = engine.rows(lo, hi, q_cap=QCAP)
    T = st.targets[1]
    sel = rows[rows["type"] == 1]
    allq = _primes_below(QCAP)
    cols = allq[allq <= T]
    rc, got = _noalloc(L, sel["p"], hi, T, cols)
    assert rc == 0
    assert np.array_equal(got[:, 0], sel["s0"]) and np.array_equal(got[:, 1], sel["s1"])
    # more rows than the fixed scratch holds: rejected, nothing launched
    too_many = np.full(4097, 1000003, dtype=np.uint64)
    rc, _ = _noalloc(L, too_many, 2 * 10**6, 10**5, cols[:10])
    assert rc == -9
    assert L.wl_strerror(rc) != b"unknown error"


def test_noalloc_no_columns_and_full_rows(engine):
    L = wl.load_library()
    # no columns: an empty product (1 = s0 + p*s1 with s0 = 1, s1 = 0), as
    # wl_rows gives with q_cap = 2
    lo, hi = 10**9, 10**9 + 200000
    rows0, st0 = engine.rows(lo, hi, q_cap=2)
    sel0 = rows0[rows0["type"] == 0][:300]
    rc, got = _noalloc(L, sel0["p"], hi, st0.targets[0], np.zeros(0, dtype=np.uint32))
    assert rc == 0
    assert np.array_equal(got[:, 0], sel0["s0"]) and np.array_equal(got[:, 1], sel0["s1"])
    assert (got[:, 0] == 1).all() and (got[:, 1] == 0).all()
    # the largest row count the scratch holds: the split count is clipped by
    # the partial-product region, which is then fullest
    rows, st = engine.rows(lo, hi, q_cap=QCAP)
    T = st.targets[0]
    sel = rows[rows["type"] == 0][:4096]
    assert len(sel) == 4096
    allq = _primes_below(QCAP)
    cols = allq[allq <= T]
    rc, got = _noalloc(L, sel["p"], hi, T, cols)
    assert rc == 0
    assert np.array_equal(got[:, 0], sel["s0"]) and np.array_equal(got[:, 1], sel["s1"])


def test_noalloc_flags_inputs_that_break_the_contract(engine):
    L = wl.load_library()
    lo, hi = 10**9, 10**9 + 20000
    rows, st = engine.rows(lo, hi, q_cap=QCAP)
    T = st.targets[0]
    sel = rows[rows["type"] == 0]
    allq = _primes_below(QCAP)
    cols = allq[allq <= T]
    bad = np.array(sel["p"], dtype=np.uint64)
    bad[3] = hi + 2          # not below p_bound
    bad[5] = 1000000000      # even
    rc, got = _noalloc(L, bad, hi, T, cols)
    assert rc == 0
    flagged = np.zeros(len(bad), dtype=bool)
    flagged[[3, 5]] = True
    assert (got[flagged] == np.uint64(0xFFFFFFFFFFFFFFFF)).all()
    assert np.array_equal(got[~flagged, 0], sel["s0"][~flagged])
    assert np.array_equal(got[~flagged, 1], sel["s1"][~flagged])
    # columns out of order, or above T: every row is flagged
    for cc in (cols[::-1].copy(), np.append(cols, np.uint32(T + 2))):
        rc, got = _noalloc(L, sel["p"], hi, T, cc)
        assert rc == 0
        assert (got == np.uint64(0xFFFFFFFFFFFFFFFF)).all()
    # and a correct call right after gives the rows again
    rc, got = _noalloc(L, sel["p"], hi, T, cols)
    assert rc == 0 and np.array_equal(got[:, 0], sel["s0"]) and np.array_equal(got[:, 1], sel["s1"])
