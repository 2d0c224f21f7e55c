"""Dense split boundaries on the CPU (clwilson_b200/csrc/wl_plan.h).

The boundaries must be strictly increasing and fall at equal shares of the
cost model's cumulative cost, also when a bucket has many more dense splits
than the cost grid has points (about 14,000 splits against 2,048 points for
the batched workload's 4-limb buckets): boundaries snapped to grid points
there left empty splits next to ones many times too long."""
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
    out = subprocess.run([driver, repr(T), repr(qd), str(Sd)], capture_output=True, text=True, check=True).stdout
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
