"""Builds the CUDA library in-tree: analyticalreconbigpatient_b200/libhelixrecon.so.

nvcc compiles every source for sm_100a only (``-gencode arch=compute_100a,
code=sm_100a``); host code goes through the system g++ with -O3 and IEEE
semantics (no fast-math), which the bit-exact host geometry tables rely on.
Usage: ``python -m analyticalreconbigpatient_b200.build [--force]``.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libhelixrecon.so")
BUILD_DIR = os.path.join(PKG, "_build")

SOURCES = ["status.cpp", "capi.cpp", "recon.cpp", "rebin.cu", "filter.cu", "bp.cu", "bp_fast.cu", "filter_tc.cu", "slab.cu", "batch.cpp", "cnn.cu", "segment.cpp", "util.cu", "phantom.cu", "probe.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-fno-fast-math", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "helixrecon.h"))
    objs = []
    nvcc = _nvcc()
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path, *headers]):
            lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, *lang, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
    if force or _stale(LIB, objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
