"""The reference's seven self-test ranges (run_test, cl_wilson.cpp:1998-2139) on the GPU.

Each case checks what the reference checks: the number of result lines, the
checksum, pi(maxtarget) (the count of sieving primes up to the largest class
target: the reference's `totalcount - prpsremoved`), and the last result's
prime and signed value.  Cases 1-4 and 7 have class targets up to 8.8e12 and
exercise the columns above 2^32; 5 and 6 are the CPU-runnable ones.
Also runs the `clwilson -s` command-line self test once.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("case", [1, 2, 3, 4, 5, 6, 7])
def test_selftest_case(engine, golden, case):
    k = golden["kat"][case - 1]
    res = engine.search(k["pmin"], k["pmax"])
    assert len(res.results) == k["results"]
    assert "%016X" % res.checksum == k["checksum"]
    assert res.stats.pi_maxtarget == k["pi_maxtarget"]
    assert res.results[-1] == (k["last_prime"], k["last_value"])


def test_cli_search_writes_reference_results_file(tmp_path):
    exe = os.path.join(ROOT, "clwilson_b200", "clwilson")
    out = subprocess.run([exe, "-p", "200", "-P", "564"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    text = (tmp_path / "results.txt").read_text().splitlines()
    assert len(text) == 58 and text[-1] == "00000000000080A3" and text[-2] == "563 is a Wilson prime"
    assert "checksum 00000000000080A3" in out.stdout


def test_cli_self_test(tmp_path):
    # `clwilson -s`: run_test's seven ranges with their checksums (cl_wilson.cpp:1998-2139)
    exe = os.path.join(ROOT, "clwilson_b200", "clwilson")
    out = subprocess.run([exe, "-s"], cwd=tmp_path, capture_output=True, text=True, timeout=900)
    assert out.returncode == 0, out.stdout + out.stderr
    assert out.stdout.count("passed.") == 7 and "All test cases completed successfully!" in out.stdout


def _good_results_file(path, lines):
    # goodWilsonResults.txt lines "p v"; the file's sum of p + v must be the
    # reference's constant (cl_wilson.cpp:970), so one balancing line far
    # above every search range closes it
    magic = 0x6659912234F44428
    s = sum(p + v for p, v in lines) % (1 << 64)
    bal = (magic - s) % (1 << 64)
    assert bal > 10**14
    path.write_text("".join(f"{p} {v}\n" for p, v in lines) + f"{bal} 0\n")


def test_cli_result_verification(tmp_path):
    # -r: the results with |w_p/p| < 1/50000 against goodWilsonResults.txt
    # (cl_wilson.cpp:902-1014); in [200, 564) that is the Wilson prime 563
    exe = os.path.join(ROOT, "clwilson_b200", "clwilson")
    _good_results_file(tmp_path / "goodWilsonResults.txt", [(563, 0)])
    out = subprocess.run([exe, "-r", "-p", "200", "-P", "564"], cwd=tmp_path, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "p: 563 has matching result +0" in out.stdout and "All results matched result file!" in out.stdout
    # a wrong value in the file is reported and fails the run
    _good_results_file(tmp_path / "goodWilsonResults.txt", [(563, 5)])
    for f in ("stateA.ckp", "stateB.ckp"):
        if (tmp_path / f).exists():
            (tmp_path / f).unlink()
    out = subprocess.run([exe, "-r", "-p", "200", "-P", "564"], cwd=tmp_path, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode != 0 and "result check failed" in out.stdout
