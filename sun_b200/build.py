"""Build ``sun_b200/libsun_b200.so`` for sm_100a with nvcc (in-tree).

The per-N kernel translation units compile in parallel; objects land in
``sun_b200/_build`` and are reused while their sources are unchanged.
``python -m sun_b200.build`` or ``__graft_entry__.build()`` run it.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsun_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no implicit multiply-add contraction; the kernels write out
# every fused operation (sun_math.cuh), so equal source arithmetic rounds
# equally in every kernel
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
              "-I" + os.path.join(ROOT, "include")] + ARCH
UNITS = ["ops_n2.cu", "ops_n3.cu", "ops_n4.cu", "ops_n6.cu", "engine.cu", "server.cu", "noalloc.cu",
         "draw_check.cu"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + _headers())


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    if not _stale(obj, src):
        return obj
    cmd = [_nvcc()] + NVCC_FLAGS + ["-c", src, "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    os.replace(obj + ".tmp", obj)
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(CSRC, u) for u in UNITS]
    jobs = jobs or min(len(srcs), max(1, os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [_nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB + ".tmp"] + objs
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
