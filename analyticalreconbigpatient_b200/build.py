"""Builds the CUDA library in-tree: analyticalreconbigpatient_b200/libhelixrecon.so.

nvcc compiles every source for sm_100a only (``-gencode arch=compute_100a,
code=sm_100a``); host code goes through the system g++ with -O3 and IEEE
semantics (no fast-math), which the bit-exact host geometry tables rely on.
Objects and libraries are rebuilt whenever the content digest of their inputs
(source, headers, compiler command) differs from the one recorded beside them.
Usage: ``python -m analyticalreconbigpatient_b200.build [--force]``.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libhelixrecon.so")
BUILD_DIR = os.path.join(PKG, "_build")

SOURCES = ["status.cpp", "capi.cpp", "recon.cpp", "rebin.cu", "filter.cu", "bp.cu", "bp_fast.cu", "filter_tc.cu", "slab.cu", "batch.cpp", "cnn.cu", "segment.cpp", "util.cu", "phantom.cu"]
# The measurement probe (the texture units' sample rate, the texture backprojection's roofline) is a
# library of its own, outside the product's C ABI.
PROBE_SOURCES = ["probe.cu", "status.cpp"]
PROBE_LIB = os.path.join(PKG, "libhelixprobe.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O3,-fno-fast-math", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return "nvcc"


def _digest(parts) -> str:
    h = hashlib.sha256()
    for part in parts:
        h.update(part if isinstance(part, bytes) else str(part).encode())
        h.update(b"\0")
    return h.hexdigest()


def _read(path: str) -> bytes:
    with open(path, "rb") as f:
        return f.read()


def _up_to_date(target: str, digest: str) -> bool:
    """A target is reused only if it exists and was built from inputs with the
    same content digest (sources, headers, flags), whatever the files' times."""
    stamp = target + ".sha256"
    return os.path.exists(target) and os.path.exists(stamp) and _read(stamp).decode().strip() == digest


def _stamp(target: str, digest: str) -> None:
    with open(target + ".sha256", "w") as f:
        f.write(digest + "\n")


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh")))
    headers.append(os.path.join(INCLUDE, "helixrecon.h"))
    header_bytes = [_read(h) for h in headers]
    nvcc = _nvcc()
    obj_digest = {}
    for src in dict.fromkeys(SOURCES + PROBE_SOURCES):
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src + ".o")
        lang = ["-x", "cu"] if src.endswith(".cu") else ["-x", "c++"]
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, *lang, "-c", path, "-o", obj]
        digest = _digest([*cmd, _read(path), *header_bytes])
        obj_digest[src] = digest
        if force or not _up_to_date(obj, digest):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            _stamp(obj, digest)
    for target, srcs in ((LIB, SOURCES), (PROBE_LIB, PROBE_SOURCES)):
        tobjs = [os.path.join(BUILD_DIR, src + ".o") for src in srcs]
        cmd = [nvcc, *ARCH, "-shared", "-o", target, *tobjs, "-lcudart"]
        digest = _digest([*cmd, *(obj_digest[src] for src in srcs)])
        if force or not _up_to_date(target, digest):
            if verbose:
                print(" ".join(cmd), flush=True)
            subprocess.run(cmd, check=True)
            _stamp(target, digest)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
