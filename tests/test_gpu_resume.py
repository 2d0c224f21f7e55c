"""Searches in pieces, checkpoints and resume (cl_wilson.cpp:110-288, 1742-1776).

* wl_rows_from / wl_search_from: the column product split at arbitrary
  sieving-prime bounds (below and above 2^32, inside the dense region)
  continues to the same rows, result lines and checksum as one call.
* The command line writes stateA.ckp / stateB.ckp in the reference's format,
  resumes from them after an interruption, reports a finished workunit, and
  resumes from a checkpoint built the way the reference program writes it
  (running products in Montgomery form with R = 2^64, kernels/common.cl:120-130).
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import clwilson_b200 as wl
import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "clwilson_b200", "clwilson")


def _pieces(engine, lo, hi, bounds, q_cap=0):
    rows = None
    q = 2
    for b in bounds:
        rows, _ = engine.rows_from(lo, hi, q, b, init=rows)
        q = b
    return engine.rows_from(lo, hi, q, q_cap, init=rows)[0], rows, q


@pytest.mark.parametrize("lo,hi,bounds", [
    (10**6, 10**6 + 5000, [1000, 50_001, 200_003]),
    (2**31 - 1000, 2**31 + 1000, [7, 2**20 + 1, 2**29]),
])
def test_full_search_in_pieces(engine, lo, hi, bounds):
    want, _ = engine.rows(lo, hi)
    got, rows, q = _pieces(engine, lo, hi, bounds)
    for f in ("p", "s0", "s1", "rem", "quot"):
        assert np.array_equal(got[f], want[f]), f
    one = engine.search(lo, hi)
    last = engine.search_from(lo, hi, q, init=rows)
    assert last.checksum == one.checksum and last.results == one.results


def test_capped_pieces_dense_and_above_2_32(engine):
    # p ~ 1e13: the columns below 2^22 are all in the dense regime; the bound
    # 2^32 + 2^25 + 12345 is inside a window of the sieve above 2^32
    lo, hi = 10**13, 10**13 + 2000
    cap = (1 << 32) + (1 << 26)
    want, _ = engine.rows(lo, hi, q_cap=cap)
    got, _, _ = _pieces(engine, lo, hi, [3_000_017, (1 << 22) + 1, (1 << 32) + (1 << 25) + 12345], q_cap=cap)
    assert np.array_equal(got["s0"], want["s0"]) and np.array_equal(got["s1"], want["s1"])


def test_kat1_in_pieces(engine, golden):
    # self-test case 1 (class targets up to 2.07e11) split below and above 2^32
    k = golden["kat"][0]
    lo, hi = k["pmin"], k["pmax"]
    rows = None
    q = 2
    for b in [(1 << 32) - 5, (1 << 32) + 12345, 5 * 10**10 + 1]:
        rows, _ = engine.rows_from(lo, hi, q, b, init=rows)
        q = b
    res = engine.search_from(lo, hi, q, init=rows)
    assert "%016X" % res.checksum == k["checksum"]
    assert res.results == [(k["last_prime"], k["last_value"])]


def _expected_results_file(engine, lo, hi):
    r = engine.search(lo, hi)
    lines = [wl.result_line(p, v) for p, v in r.results]
    lines.append("%016X" % r.checksum if r.results else "no results\n%016X" % r.checksum)
    return "\n".join(lines) + "\n"


def _run(cwd, lo, hi, **env):
    e = dict(os.environ)
    e.update({k: str(v) for k, v in env.items()})
    return subprocess.run([EXE, "-p", str(lo), "-P", str(hi)], cwd=cwd, env=e, capture_output=True, text=True,
                          timeout=600)


def test_cli_interrupt_and_resume(engine, tmp_path):
    lo, hi = 10**6, 10**6 + 20000
    want = _expected_results_file(engine, lo, hi)
    # pieces of 100,000 integers, stopped after two: a checkpoint, no results yet
    out = _run(tmp_path, lo, hi, WL_CKPT_PIECE=100000, WL_CKPT_STOP=2)
    assert out.returncode == 3, out.stdout + out.stderr
    assert (tmp_path / "stateA.ckp").exists()
    hdr = (tmp_path / "stateA.ckp").read_bytes()[:56]
    pmin, pmax, currp, trickle, ssum, total, tpcount, done = struct.unpack("<6Q2I", hdr)
    assert (pmin, pmax, currp, done) == (lo, hi, 200002, 0)
    # resumed, finished in pieces
    out = _run(tmp_path, lo, hi, WL_CKPT_PIECE=100000)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "Resuming search from checkpoint. Current P: 200002" in out.stdout
    assert (tmp_path / "results.txt").read_text() == want
    # the finished workunit is reported, not searched again
    out = _run(tmp_path, lo, hi)
    assert out.returncode == 0 and "Workunit complete." in out.stdout


def _to_reference(p, v):
    n = p * p
    r = (v << 64) % n
    return r % p, r // p


def test_cli_resumes_reference_checkpoint(tmp_path, engine):
    # a stateB.ckp as the reference writes it: the running products over the
    # sieving primes below currp (here from the oracle), Montgomery form R = 2^64
    lo, hi = 10**6, 10**6 + 3000
    currp = 150_001
    rows, _ = oracle.search(lo, hi, qcap=currp)
    res = []
    for r in rows:
        p = int(r["p"])
        res += list(_to_reference(p, int(r["s0"]) + p * int(r["s1"])))
    trickle, total, tpcount = 1234567, 13848, len(rows)
    ssum = (lo + hi + currp + trickle + total + tpcount + 0 + sum(res)) % (1 << 64)
    data = struct.pack("<6Q2I", lo, hi, currp, trickle, ssum, total, tpcount, 0)
    data += struct.pack("<%dQ" % len(res), *res)
    (tmp_path / "stateB.ckp").write_bytes(data)
    # a corrupt stateA.ckp is rejected by its checksum
    bad = bytearray(data)
    bad[-1] ^= 1
    (tmp_path / "stateA.ckp").write_bytes(bytes(bad))
    out = _run(tmp_path, lo, hi)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "Checksum error in stateA.ckp" in out.stdout
    assert "Resuming search from checkpoint. Current P: 150001" in out.stdout
    assert (tmp_path / "results.txt").read_text() == _expected_results_file(engine, lo, hi)
