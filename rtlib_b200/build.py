"""Build recipe of the rtlib_b200 native library (nvcc, sm_100a only).

Produces rtlib_b200/librtpg.so in-tree.  Every .cu file under csrc/ is compiled for
``-gencode arch=compute_100a,code=sm_100a``.  The guiding, hash-grid, BVH and tracer
kernels are compiled with ``-fmad=false`` so every float operation rounds exactly as written
(their results are checked against the CPU oracle, bit for bit where the arithmetic allows).
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "librtpg.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "-Xcompiler", "-Wall", "--expt-relaxed-constexpr", "-DRTPG_BUILD"]
# files whose float arithmetic must round as written (bit-exact parity with the oracle)
EXACT = {"sdtree.cu", "common.cu", "hashgrid.cu", "mqt.cu", "tracer.cu", "bvh.cu"}


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))


def _needs(obj, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "rtpg.h"))
    objs = []
    for f in sources():
        src = os.path.join(CSRC, f)
        obj = os.path.join(BUILD, f[:-3] + ".o")
        objs.append(obj)
        if not force and not _needs(obj, [src] + headers):
            continue
        flags = ["-fmad=false"] if f in EXACT else []
        cmd = [NVCC, *ARCH, *COMMON, *flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    if force or _needs(OUT, objs):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", *objs, "-o", OUT, "-lcudart_static", "-lrt",
               "-lpthread", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return OUT


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv)
