"""The serving row pool on the CPU (clwilson_b200/csrc/wl_pool.h): first-fit
allocation of contiguous row ranges and coalescing releases, under random
sequences of requests of mixed sizes, against an explicit row map."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("pool") / "pool_driver")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "clwilson_b200", "csrc"),
                           os.path.join(ROOT, "tests", "pool_driver.cpp"), "-o", out])
    return out


@pytest.mark.parametrize("cap,ops,seed", [(5000, 20000, 1), (300, 20000, 2), (64, 20000, 3)])
def test_random_sequences(driver, cap, ops, seed):
    r = subprocess.run([driver, str(cap), str(ops), str(seed)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("ok"), r.stdout + r.stderr
