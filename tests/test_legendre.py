"""The column exponent v_q(T!) (Legendre's formula) on the host, against Python integers.

legendre() (clwilson_b200/csrc/wl_arith.cuh) gives every sweep its column
exponents: sum over k of floor(T / q^k), the reference's getPower
(cl_wilson.cpp:1293-1313).  It forms the terms as running quotients and
switches to 32-bit division once a quotient and q fit 32 bits, so the cases
below sit on those edges: quotients just below and above 2^32, q just below
and above 2^32 (the columns above the resident table), q^2 and q^3 around T,
q above T, and targets up to the top of the range (p < 2^62, T = (p-1)/2).
The function is also a host function; this compiles it with nvcc for the CPU.
"""
import os
import random
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "clwilson_b200", "csrc")

PROGRAM = r"""
#include <cstdio>
#include "wl_arith.cuh"
int main() {
    unsigned long long T, q;
    while (scanf("%llx %llx", &T, &q) == 2) printf("%llx\n", (unsigned long long)wl::legendre(T, q));
    return 0;
}
"""


def _exact(T, q):
    e, qq = 0, q
    while qq <= T:
        e += T // qq
        qq *= q
    return e


def _cases(rng):
    out = []
    top = (1 << 61) - 1                                  # (2^62 - 2) / 2
    for q in (2, 3, 5, 7, 65521, (1 << 31) - 1, (1 << 32) - 5, (1 << 32) + 15, (1 << 33) + 17):
        for T in (0, 1, q - 1, q, q + 1, q * q - 1, q * q, q * q * q, top, top - 1):
            if T <= top:
                out.append((T, q))
        # quotients T / q^k right at 2^32
        for k in (1, 2):
            for d in (-1, 0, 1):
                T = ((1 << 32) + d) * q ** k
                if 0 <= T <= top:
                    out.append((T, q))
    for _ in range(4000):
        q = rng.choice([rng.randrange(2, 1 << 16), rng.randrange(1 << 16, 1 << 32), rng.randrange(1 << 32, 1 << 34)])
        T = rng.choice([rng.randrange(0, top), rng.randrange(0, 1 << 40), q * q + rng.randrange(-q, q)])
        out.append((max(0, min(T, top)), q))
    return out


@pytest.fixture(scope="module")
def legendre_prog(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("legendre")
    src = d / "legendre.cu"
    src.write_text(PROGRAM)
    exe = d / "legendre"
    subprocess.check_call([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets",
                           "-I", os.path.join(ROOT, "include"), "-I", CSRC, str(src), "-o", str(exe)])
    return str(exe)


def test_legendre_against_integers(legendre_prog):
    cases = _cases(random.Random(20261205))
    inp = "".join("%x %x\n" % (T, q) for T, q in cases)
    out = subprocess.run([legendre_prog], input=inp, capture_output=True, text=True, check=True).stdout.split()
    assert len(out) == len(cases)
    for (T, q), got in zip(cases, out):
        assert int(got, 16) == _exact(T, q), (hex(T), hex(q))
