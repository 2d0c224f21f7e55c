"""The capped sweeps of the mid-size and top-of-range workloads, pinned to the oracle.

The plain-mid ([1e13, 1e13+1e7)) and plain-top ([2^62-1-1e7, 2^62-1))
workloads run with every column q < 2^32.  For sampled rows of each, this
checks the product over column windows that only those caps reach:

* [2^31, 2^31 + 2^26): columns of 32 bits whose cell needs the conditional
  subtraction (q >= 2^31) on 3- and 4-limb rows;
* [2^32 - 2^26, 2^32): the last columns of the resident table;
* a window in the dense regime (exponents change at nearly every column):
  around 2^24 for p near 2^62, below 2^22.7 for p near 1e13.

Two ways per window [a, b):
* capped(b) = capped(a) * W mod p^2, where capped(x) is the engine's capped
  sweep over q < x (the bench's call) and W the oracle's product
  prod_{a <= q < b} q^{v_q(T!)} (mullarge.cl:36-63, mulsmall.cl:32-58);
* the engine's piece over [a, b) alone (wl_rows_from) equals W.
"""
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

MID = (10**13, 10**13 + 20000)
TOP = ((1 << 62) - 1 - 20000, (1 << 62) - 1)
WINDOWS = {
    "q>=2^31": (1 << 31, (1 << 31) + (1 << 26)),
    "below 2^32": ((1 << 32) - (1 << 26), 1 << 32),
    "dense 2^24": ((1 << 24) - (1 << 22), (1 << 24) + (1 << 22)),
    "dense 2^21": (1 << 21, (1 << 21) + (1 << 21)),
}
CASES = [(MID, "q>=2^31"), (MID, "below 2^32"), (MID, "dense 2^21"),
         (TOP, "q>=2^31"), (TOP, "below 2^32"), (TOP, "dense 2^24")]


def _oracle_window(args):
    p, T, a, b = args
    return oracle.range_product(p, T, a, b)


def _sample(rows, k=4):
    # rows of every class first, then evenly spaced ones
    idx = []
    for t in (0, 1, 2):
        hit = np.nonzero(rows["type"] == t)[0]
        if hit.size:
            idx.append(int(hit[hit.size // 2]))
    for i in np.linspace(0, len(rows) - 1, k).astype(int):
        if len(idx) >= k:
            break
        if int(i) not in idx:
            idx.append(int(i))
    return idx[:k]


@pytest.fixture(scope="module")
def oracle_built():
    oracle.build()


@pytest.mark.parametrize("rng,win", CASES, ids=["%s-%s" % ("mid" if r is MID else "top", w) for r, w in CASES])
def test_capped_window_against_oracle(engine, oracle_built, rng, win):
    lo, hi = rng
    a, b = WINDOWS[win]
    ra, st = engine.rows(lo, hi, q_cap=a)
    rb, _ = engine.rows(lo, hi, q_cap=b)
    piece, _ = engine.rows_from(lo, hi, a, b)
    assert np.array_equal(ra["p"], rb["p"]) and np.array_equal(ra["p"], piece["p"])
    idx = _sample(ra)
    if win.startswith("dense"):
        # the window lies where floor(T/q) drops at nearly every prime
        # (T ln q / q^2 > 1), the dense sweep's regime
        assert min(t for t in st.targets if t) * 14 > b * b
    jobs = [(int(ra["p"][i]), st.targets[int(ra["type"][i])], a, b) for i in idx]
    with ThreadPoolExecutor(max_workers=8) as ex:
        want = list(ex.map(_oracle_window, jobs))
    for i, (w0, w1) in zip(idx, want):
        p = int(ra["p"][i])
        m = p * p
        x = int(ra["s0"][i]) + p * int(ra["s1"][i])
        y = int(rb["s0"][i]) + p * int(rb["s1"][i])
        w = w0 + p * w1
        assert x * w % m == y, (p, win)
        assert (int(piece["s0"][i]), int(piece["s1"][i])) == (w0, w1), (p, win)
