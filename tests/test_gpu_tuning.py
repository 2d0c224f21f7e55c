"""Kernel tuning (wl_autotune, wl_get_tuning, wl_set_tuning).

Every variant the tuner may choose gives the same rows: checked on capped
golden vectors (dense regime at p ~ 1e13 and 2^62) and a full search, with
each dense kernel, each prefix-fold cell formulation and rows-per-thread
setting, and each merge fan-in.
"""
import numpy as np
import pytest

import clwilson_b200 as wl
import oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big_rows():
    # about 2,200 primes: buckets of more than 512 rows take the two-rows-per-thread sweep
    oracle.build()
    rows, _ = oracle.search(10**6, 10**6 + 30000)
    return rows


@pytest.fixture(scope="module")
def eng():
    e = wl.Engine(0)
    yield e
    e.close()


def _capped_ok(e, golden, lo, hi, qcap):
    case = next(c for c in golden["capped"] if c["pmin"] == lo)
    rows, _ = e.rows(lo, hi, q_cap=qcap)
    byp = {int(p): i for i, p in enumerate(rows["p"])}
    for w in case["rows"]:
        r = rows[byp[w["p"]]]
        assert (int(r["s0"]), int(r["s1"])) == (w["s0"], w["s1"]), w["p"]


@pytest.mark.parametrize("kernel", [0, 1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("hstep", [4, 16])
def test_dense_variants(eng, golden, kernel, hstep):
    eng.tuning = {"dense_kernel": [kernel] * 3, "dense_hstep": [hstep] * 3}
    _capped_ok(eng, golden, 10**13, 10**13 + 10**7, 1 << 16)
    _capped_ok(eng, golden, (1 << 62) - 1 - 10**7, (1 << 62) - 1, 1 << 16)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
@pytest.mark.parametrize("rpt", [1, 2, 4])
@pytest.mark.parametrize("merge", [1, 10**6])
def test_sparse_variants_full_search(eng, golden, big_rows, variant, rpt, merge):
    eng.tuning = {"sparse_variant": [variant] * 3, "sparse_rpt": [rpt] * 3, "merge_cta_min": merge,
                  "dense_kernel": [0] * 3, "dense_hstep": [8] * 3}
    rows, _ = eng.rows(10**6, 10**6 + 30000)
    for f in ("p", "s0", "s1", "rem", "quot"):
        assert np.array_equal(rows[f].astype(np.uint64), big_rows[f].astype(np.uint64)), f
    g = golden["range_1e5"]
    res = eng.search(g["pmin"], g["pmax"])
    assert res.lines() == g["lines"] and "%016X" % res.checksum == g["checksum"]
    k = golden["kat"][4]
    res = eng.search(k["pmin"], k["pmax"])
    assert "%016X" % res.checksum == k["checksum"]


def test_set_tuning_rejects_bad_values(eng):
    with pytest.raises(wl.WilsonError):
        eng.tuning = {"dense_kernel": [7, 0, 0]}
    with pytest.raises(wl.WilsonError):
        eng.tuning = {"sparse_rpt": [3, 1, 1]}
    with pytest.raises(wl.WilsonError):
        eng.tuning = {"sparse_variant": [4, 1, 1]}


def test_autotune_and_serving_with_tuning(eng):
    t = eng.autotune([(10**9, 10**9 + 100000)])
    # any of the sparse cell formulations (0-3) may win on this box
    assert t["ms"][0] > 0 and t["sparse_variant"][0] in (0, 1, 2, 3) and t["dense_kernel"][0] in range(7)
    assert eng.tuning == t
    t2 = eng.autotune(limbs=(4,))                      # built-in sample
    assert t2["ms"][2] > 0
    want = eng.search(10**6, 10**6 + 3000)
    with wl.Server(0, tuning=t) as srv:
        info = srv.wait(srv.submit(10**6, 10**6 + 3000), 600_000)
        assert info.state == "done" and info.checksum == want.checksum
