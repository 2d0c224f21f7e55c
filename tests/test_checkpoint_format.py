"""The checkpoint files on the CPU (clwilson_b200/csrc/wl_ckpt.h).

Byte layout of the reference's workStatus header and residues
(cl_wilson.h:22-25, cl_wilson.cpp:110-152), its additive state_sum, the
choice of the newer valid file of stateA/stateB (159-288), and the conversion
between plain values and the reference's Montgomery digits (R = 2^64 mod p^2,
kernels/common.cl:120-130), checked against Python integers.
"""
import os
import random
import struct
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = "<6Q2I"


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("ckpt") / "ckpt_driver")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "clwilson_b200", "csrc"),
                           os.path.join(ROOT, "tests", "ckpt_driver.cpp"), "-o", out])
    return out


def _run(driver, cwd, *args):
    r = subprocess.run([driver, *map(str, args)], cwd=cwd, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def test_reference_montgomery_digits(driver, tmp_path):
    rng = random.Random(7)
    primes = [5, 563, 1000000007, 4294967291] + [p for p in oracle.list_primes((1 << 62) - 2000, (1 << 62) - 1)[:3]]
    for p in map(int, primes):
        n = p * p
        for _ in range(5):
            v = rng.randrange(n)
            r0, r1, s0, s1 = map(int, _run(driver, tmp_path, "conv", p, v % p, v // p).split())
            r = (v << 64) % n
            assert (r0, r1) == (r % p, r // p), p
            assert (s0, s1) == (v % p, v // p), p


def _residues(k):
    return [1000 + i for i in range(2 * k)]


def test_write_layout_and_checksum(driver, tmp_path):
    res = _residues(3)
    out = _run(driver, tmp_path, "write", "A", 200, 564, 101, 1234, 26, 0, *res)
    assert out.strip() == "next B"
    data = (tmp_path / "stateA.ckp").read_bytes()
    assert len(data) == 56 + 16 * 3
    pmin, pmax, currp, trickle, ssum, total, tpcount, done = struct.unpack(HDR, data[:56])
    assert (pmin, pmax, currp, trickle, total, tpcount, done) == (200, 564, 101, 1234, 26, 3, 0)
    assert ssum == (200 + 564 + 101 + 1234 + 26 + 3 + 0 + sum(res)) % (1 << 64)
    assert list(struct.unpack("<6Q", data[56:])) == res


def test_newest_valid_file_wins(driver, tmp_path):
    _run(driver, tmp_path, "write", "A", 200, 564, 101, 1, 0, 0, *_residues(2))
    _run(driver, tmp_path, "write", "B", 200, 564, 307, 1, 0, 0, *[7, 8, 9, 10])
    out = _run(driver, tmp_path, "read", 200, 564, 2)
    assert out.split()[:5] == ["status", "1", "currp", "307", "next"] and out.split()[5] == "A"
    assert out.split()[6:] == ["7", "8", "9", "10"]
    # a corrupt B: its checksum fails, A is used and B is written next
    b = bytearray((tmp_path / "stateB.ckp").read_bytes())
    b[-1] ^= 1
    (tmp_path / "stateB.ckp").write_bytes(bytes(b))
    out = _run(driver, tmp_path, "read", 200, 564, 2)
    assert "Checksum error in stateB.ckp" in out
    assert out.splitlines()[-1].split()[:6] == ["status", "1", "currp", "101", "next", "B"]
    # a checkpoint of another range is rejected
    out = _run(driver, tmp_path, "read", 200, 600, 2)
    assert "Invalid checkpoint file" in out and out.splitlines()[-1].startswith("status 0")
    # a finished workunit
    _run(driver, tmp_path, "write", "B", 200, 564, 400, 1, 0, 1, *_residues(2))
    assert _run(driver, tmp_path, "read", 200, 564, 2).splitlines()[-1].startswith("status 2")


def test_files_past_2_32(driver, tmp_path):
    # p ~ 1e10: the type-2 target (p-1)/2 is above 2^32, so a search checkpoints
    # past 2^32, where the reference's running products hold base-2
    # pseudoprime factors (cl_wilson.cpp:709-726) and this program's do not
    lo, hi = 10**10, 10**10 + 200
    past = (1 << 32) + 1001
    # a file of this program past 2^32 goes to its own name, and resumes
    out = _run(driver, tmp_path, "write", "A", lo, hi, past, 1, 0, 0, *_residues(2))
    assert out.strip() == "next B"
    assert (tmp_path / "stateA.b200.ckp").exists() and not (tmp_path / "stateA.ckp").exists()
    out = _run(driver, tmp_path, "read", lo, hi, 2)
    assert out.split()[:4] == ["status", "1", "currp", str(past)]
    # a reference-named file at currp = 2^32 is shared by both programs
    d2 = tmp_path / "shared"
    d2.mkdir()
    _run(driver, d2, "write", "B", lo, hi, 1 << 32, 1, 0, 0, *_residues(2))
    assert (d2 / "stateB.ckp").exists()
    out = _run(driver, d2, "read", lo, hi, 2)
    assert out.split()[:4] == ["status", "1", "currp", str(1 << 32)]
    # a reference-named file past 2^32 (as the reference writes it) is refused
    # with a message, also when an older file of this program exists
    data = bytearray((tmp_path / "stateA.b200.ckp").read_bytes())
    pmin, pmax, currp, trickle, ssum, total, tpcount, done = struct.unpack(HDR, bytes(data[:56]))
    currp2 = past + 10**6
    ssum2 = (ssum - currp + currp2) % (1 << 64)
    data[:56] = struct.pack(HDR, pmin, pmax, currp2, trickle, ssum2, total, tpcount, done)
    (tmp_path / "stateB.ckp").write_bytes(bytes(data))
    out = _run(driver, tmp_path, "read", lo, hi, 2)
    assert "past 2^32" in out and "stateB.ckp" in out
    assert out.splitlines()[-1].startswith("status 3")
    # a finished workunit is reported whatever its currp
    _run(driver, tmp_path, "write", "A", lo, hi, past + 5, 1, 0, 1, *_residues(2))
    assert (tmp_path / "stateA.ckp").exists()
    assert _run(driver, tmp_path, "read", lo, hi, 2).splitlines()[-1].startswith("status 2")
