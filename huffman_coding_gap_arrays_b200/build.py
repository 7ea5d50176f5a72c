"""Builds libhgap.so in-tree with nvcc for sm_100a.

    python -m huffman_coding_gap_arrays_b200.build

Objects go to ``_build/`` at the repository root (git-ignored); the shared
library lands next to this file so it travels with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "hgap")
LIB = os.path.join(PKG, "libhgap.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2,-Wall",
         "-Wno-deprecated-gpu-targets", "-I" + os.path.join(ROOT, "include")]

SOURCES = ["hist.cu", "encode.cu", "decode.cu", "api.cu", "batch.cu", "mlp.cu", "compat.cu", "noalloc.cu",
           "host.cpp"]
HEADERS = ["hgap_internal.h", "device_util.cuh", "book.cuh", "dec_entry.cuh", "launch_cache.h"]


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(ROOT, "include", "hgap.h")]
    objs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", s, "-o", o]
            if ptxas_info and src.endswith(".cu"):
                cmd.insert(1, "-Xptxas=-v")
            r = _run(cmd, verbose)
            if ptxas_info:
                print(r.stderr, end="")
    if force or _newer(LIB, objs):
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs], verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
