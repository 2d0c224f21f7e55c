"""The Montgomery limb step of the column groups, on the host, against Python integers.

limb_step<L> (clwilson_b200/csrc/wl_arith.cuh) multiplies a residue x < 2n by
a multi-limb multiplier W, one 32-bit limb at a time:
    t <- (t + x*w_j + m*n) / 2^32,   t = 0 before the first limb.
After k limbs t = x*W*2^(-32k) mod n, and t < x + n after every step, so one
conditional subtraction leaves it below 2n.  The function is also a host
function, so this compiles it with nvcc for the CPU and checks both facts on
moduli n = p^2 at the top of each limb width (p just below 2^31, 2^47, 2^62),
at the bottom, and at random, with limbs of all ones and of zeros among the
random ones.
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
#include <cstdlib>
#include "wl_arith.cuh"
using namespace wl;

// reads: L k n[L] ninv x[L] w[k]; prints t after every step, L limbs per line
template <int L> static void run(int k) {
    uint32_t n[L], x0[L], ninv;
    for (int i = 0; i < L; ++i) if (scanf("%x", &n[i]) != 1) exit(2);
    if (scanf("%x", &ninv) != 1) exit(2);
    Res<L> x;
    for (int i = 0; i < L; ++i) { if (scanf("%x", &x0[i]) != 1) exit(2); x.w[i] = x0[i]; }
    uint32_t t[L] = {};
    for (int j = 0; j < k; ++j) {
        uint32_t w;
        if (scanf("%x", &w) != 1) exit(2);
        limb_step<L>(t, x, w, n, ninv);
        for (int i = 0; i < L; ++i) printf("%08x%c", t[i], i + 1 < L ? ' ' : '\n');
    }
}

int main() {
    int L, k;
    while (scanf("%d %d", &L, &k) == 2) {
        if (L == 2) run<2>(k);
        else if (L == 3) run<3>(k);
        else run<4>(k);
    }
    return 0;
}
"""

TOP = {2: 1 << 31, 3: 1 << 47, 4: 1 << 62}


def _limbs(v, L):
    return [(v >> (32 * i)) & 0xFFFFFFFF for i in range(L)]


def _cases(rng):
    out = []
    for L in (2, 3, 4):
        lo = TOP[L - 1] if L > 2 else 5
        ps = [TOP[L] - 1, TOP[L] - 3, lo | 1]
        ps += [rng.randrange(lo, TOP[L]) | 1 for _ in range(12)]
        for p in ps:
            n = p * p
            ninv = (-pow(n, -1, 1 << 32)) % (1 << 32)
            for x in (2 * n - 1, 0, 1, rng.randrange(2 * n)):
                k = rng.randrange(1, 33)
                ws = [rng.choice([0xFFFFFFFF, 0, rng.getrandbits(32), rng.getrandbits(32)]) for _ in range(k)]
                out.append((L, n, ninv, x, ws))
    return out


@pytest.fixture(scope="module")
def limb_prog(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc) and not shutil.which("nvcc"):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("limb")
    src = d / "limb.cu"
    src.write_text(PROGRAM)
    exe = d / "limb"
    subprocess.check_call([nvcc, "-std=c++17", "-O2", "-Wno-deprecated-gpu-targets",
                           "-I", os.path.join(ROOT, "include"), "-I", CSRC, str(src), "-o", str(exe)])
    return str(exe)


def test_limb_step_against_integers(limb_prog):
    rng = random.Random(20261204)
    cases = _cases(rng)
    lines = []
    for L, n, ninv, x, ws in cases:
        lines.append("%d %d" % (L, len(ws)))
        lines.append(" ".join("%x" % v for v in _limbs(n, L)) + " %x" % ninv)
        lines.append(" ".join("%x" % v for v in _limbs(x, L)))
        lines.append(" ".join("%x" % w for w in ws))
    out = subprocess.run([limb_prog], input="\n".join(lines) + "\n", capture_output=True, text=True,
                         check=True).stdout.split("\n")
    pos = 0
    R = 1 << 32
    for L, n, ninv, x, ws in cases:
        W = 0
        for j, w in enumerate(ws):
            W += w << (32 * j)
            limbs = [int(v, 16) for v in out[pos].split()]
            pos += 1
            t = sum(v << (32 * i) for i, v in enumerate(limbs))
            # the running sum stays below x + n, and equals x * (limbs so far) / R^(j+1) mod n
            assert t < x + n, (L, hex(n), hex(x), j)
            assert (t * pow(R, j + 1, n) - x * W) % n == 0, (L, hex(n), hex(x), j)
        if t >= n:
            t -= n
        assert t < 2 * n
        assert t % n == x * W * pow(R, -len(ws), n) % n
