"""Build libquoin_b200.so in-tree with nvcc for sm_100a.

Every CUDA translation unit is compiled with -fmad=false: the float codecs
(ALP, FLOAT_MULT, ALP-RD's cost estimate) must reproduce IEEE doubles exactly,
as the reference computes them without contraction.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libquoin_b200.so")

SOURCES = ["qb_decode.cu", "qb_dparse.cu", "qb_encode.cu", "qb_lower.cu", "qb_noalloc.cu", "qb_host.cpp", "qb_arrow.cpp", "qb_batch.cpp",
           "qb_serve.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# Host code: POPCNT for the validity counts (every x86-64 server CPU of the
# B200 generation has it).
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-Xcompiler", "-Wall", "-Xcompiler", "-mpopcnt"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "quoin.h"))
    objs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        objs.append(obj)
        if _newer(obj, [path, *headers, __file__]):
            continue
        cmd = [NVCC, *ARCH, *FLAGS, "-c", path, "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    if not _newer(LIB, objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-cudart", "static", "-Xcompiler", "-fPIC"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, ptxas_info="--ptxas" in sys.argv)
