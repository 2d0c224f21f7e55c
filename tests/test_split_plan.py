"""Split planning on the CPU (clwilson_b200/csrc/wl_plan.h).

* Dense split boundaries are strictly increasing and fall at equal shares of
  the cost model's cumulative cost, also when a bucket has many more dense
  splits than the cost grid has points (about 14,000 splits against 2,048
  points for the batched workload's 4-limb buckets): boundaries snapped to grid
  points there left empty splits next to ones many times too long.
* Split counts keep dense splits at 256 to 1,024 columns and prefix-fold splits
  at 2,048 to 2^17 columns.
* The memory budget lengthens splits so that the partials of the full
  top-of-range workload (2.3e5 rows, 2e8 dense columns) fit; without it the
  1,024-column rule asks for about 740 GB.
* The test-prime window layout of a batch of ranges (one launch for all):
  every odd number of each range has a thread of that range's blocks, and
  the blocks stay within the range's own bitmap words and counters."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("plan") / "plan_driver")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "clwilson_b200", "csrc"),
                           os.path.join(ROOT, "tests", "plan_driver.cpp"), "-o", out])
    return out


@pytest.mark.parametrize("T,qd,Sd", [
    (2.0**60, 2.0**28, 14000),        # a batched 4-limb bucket: many more splits than grid points
    (1.7e12, 5.0e6, 400),             # plain-mid (p ~ 1e13)
    (5.0e8, 7.4e4, 64),               # plain-small, type 2
])
def test_boundaries_increase_at_equal_cost(driver, T, qd, Sd):
    out = subprocess.run([driver, "bounds", repr(T), repr(qd), str(Sd)], capture_output=True, text=True,
                         check=True).stdout
    lines = out.strip().splitlines()
    grid_n, total = int(lines[0].split()[1]), float(lines[0].split()[3])
    pts = [tuple(map(float, ln.split())) for ln in lines[1:]]
    assert len(pts) == Sd - 1
    qs = [q for q, _ in pts]
    assert all(b > a for a, b in zip(qs, qs[1:])), "boundaries must strictly increase"
    assert 2.0 <= qs[0] and qs[-1] <= qd
    for k, (_, c) in enumerate(pts, start=1):
        assert abs(c - total * k / Sd) <= 1e-6 * total, k
    if Sd > grid_n:
        # far more distinct boundaries than grid points
        assert len(set(qs)) == Sd - 1


THREADS = 148 * 2048 * 4.0


def _splits(driver, *args):
    out = subprocess.run([driver, "splits", *map(str, args)], capture_output=True, text=True, check=True).stdout
    return tuple(map(int, out.split()))


@pytest.mark.parametrize("nrows,nd,ns,share", [(48000, 0, 26_000_000, 0.5), (22, 14_000_000, 0, 0.001),
                                               (22, 400_000, 14_000_000, 0.001), (100_000, 0, 5_000, 1.0)])
def test_split_lengths(driver, nrows, nd, ns, share):
    dcost = 5.0 * nd
    W = (nrows * (ns + dcost)) / share            # this bucket's share of all work
    Sd, Ss = _splits(driver, nrows, 2 if nrows >= 512 else 1, nd, ns, dcost, W, THREADS, 1.0)
    if nd:
        assert 256 <= nd / Sd <= 1024 or Sd == 1
    if ns:
        assert ns / Ss <= (1 << 17) + 1 and (ns / Ss >= 2048 or Ss == 1)
    assert Sd + Ss >= 1


def test_memory_budget_top_of_range(driver):
    # 3 buckets of the full top-of-range workload (all columns dense below 2^32)
    buckets = [(78000, 203_000_000, 0, 4.5 * 203_000_000)] * 3
    W = sum(n * (ns + dc) for n, nd, ns, dc in buckets)
    budget = 24 * 2**30 / 16
    args = [W, THREADS, budget] + [x for b in buckets for x in b]
    sc, tot = map(float, subprocess.run([driver, "scale", *map(str, args)], capture_output=True, text=True,
                                        check=True).stdout.split())
    assert sc < 0.05 and tot <= budget   # about 1.6e9 partials allowed against 4.6e10 asked
    # unscaled, the 1,024-column rule alone would ask for ~740 GB of partials
    Sd, _ = _splits(driver, 78000, 2, 203_000_000, 0, 4.5 * 203_000_000, W, THREADS, 1.0)
    assert Sd * 78000 * 3 * 16 > 700e9


def _windows(driver, ranges, span=1 << 18):
    args = [driver, "windows", str(span)]
    for lo, hi in ranges:
        args += [str(lo), str(hi)]
    lines = subprocess.run(args, capture_output=True, text=True, check=True).stdout.strip().splitlines()
    words, segs, blocks = map(int, lines[0].split())
    rows = [tuple(int(x) for x in ln.split()) for ln in lines[1:]]
    return words, segs, blocks, rows


def _random_ranges(seed, n):
    import numpy as np
    rng = np.random.default_rng(seed)
    starts = np.exp(rng.uniform(np.log(5.0), np.log(2.0**62 - 2e7), n))
    widths = np.exp(rng.uniform(0.0, np.log(1e7), n))
    return [(int(s), int(s) + max(1, int(w))) for s, w in zip(starts, widths)]


@pytest.mark.parametrize("ranges", [
    [(10**9, 10**9 + 10**6)],
    [(5, 6), (6, 7), (7, 8), (1 << 20, (1 << 20) + (1 << 18)), ((1 << 20) + 1, (1 << 20) + 1 + (1 << 18)),
     ((1 << 62) - 10**7, (1 << 62) - 1), (10**6, 10**6 + 1)],
    "random",
])
def test_window_layout(driver, ranges):
    # the layout of k_window_primes_multi: every odd number of a range is one
    # thread of that range's blocks, and its blocks write only that range's
    # bitmap words and segment counters, which follow the previous range's
    if ranges == "random":
        ranges = _random_ranges(7, 300)
    span = 1 << 18
    words, segs, blocks, rows = _windows(driver, ranges, span)
    assert len(rows) == len(ranges)
    w = s = b = 0
    for (lo, hi), (lo0, nseg, word_off, seg_off, block0, nblocks) in zip(ranges, rows):
        assert lo0 == lo & ~1 and (word_off, seg_off, block0) == (w, s, b)
        assert nseg * span >= hi - lo0 > (nseg - 1) * span
        # odd numbers lo0 + 2j + 1 for j < nblocks * 256: all of [lo, hi), within the segments
        first_j, last_j = (lo - lo0 - 1 + 1) // 2, (hi - 1 - lo0 - 1) // 2
        assert 0 <= first_j and last_j < nblocks * 256
        assert nblocks * 256 <= nseg * span // 2
        # ceil((hi - lo0) / 512) blocks: the last starts at most one (even) integer past the range
        assert nblocks == (hi - lo0 + 511) // 512
        assert (nblocks - 1) * 256 <= last_j + 1
        w += nseg * span // 64
        s += nseg
        b += nblocks
    assert (words, segs, blocks) == (w, s, b)
