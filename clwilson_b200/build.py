"""Build libwilson.so (CUDA, sm_100a) and the clwilson command-line binary in-tree.

    python -m clwilson_b200.build          # build if sources are newer
    python -m clwilson_b200.build --force
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libwilson.so")
CLI = os.path.join(PKG, "clwilson")

CU_SOURCES = ["wl_kernels.cu", "wl_engine.cu", "wl_serve.cu", "wl_probe.cu", "wl_noalloc.cu"]
HEADERS = ["wl_arith.cuh", "wl_internal.h", "wl_host.h", "wl_pool.h", "wl_ckpt.h", "wl_plan.h"]
NVCC_FLAGS = [
    "-O3", "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "-Xcompiler", "-fPIC",
    "-Xcompiler", "-O3",
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in CU_SOURCES + HEADERS] + [os.path.join(INCLUDE, "wilson.h"), os.path.join(INCLUDE, "wilson_probe.h")]
    if force or _stale(LIB, deps):
        objs = []
        bdir = os.path.join(PKG, "_build")
        os.makedirs(bdir, exist_ok=True)
        procs = []
        for src in CU_SOURCES:
            obj = os.path.join(bdir, src.replace(".cu", ".o"))
            cmd = [_nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-I", CSRC, "-c", os.path.join(CSRC, src), "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append(subprocess.Popen(cmd))
            objs.append(obj)
        for p in procs:
            if p.wait() != 0:
                raise RuntimeError("nvcc failed")
        tmp = LIB + ".tmp"
        cmd = [_nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", tmp, "-lcudart"]
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    cli_src = os.path.join(CSRC, "wl_cli.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB, os.path.join(INCLUDE, "wilson.h"),
                                                            os.path.join(CSRC, "wl_ckpt.h")])):
        cmd = ["g++", "-O2", "-std=c++17", "-I", INCLUDE, "-I", CSRC, cli_src, "-o", CLI + ".tmp",
               "-L", PKG, "-lwilson", "-Wl,-rpath,$ORIGIN"]
        subprocess.check_call(cmd)
        os.replace(CLI + ".tmp", CLI)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
