"""Builds rls_b200/librls_b200.so (sm_100a) in-tree with nvcc and g++.

    python -m rls_b200.build [--force]

The grid code, the IC factorisation and the MatrixMarket reader are compiled by g++ with
-ffp-contract=off (bit-exact coordinates and factors);
the CUDA translation unit by nvcc for sm_100a only.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "librls_b200.so")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cuh", ".cpp", ".h")):
            out.append(os.path.join(CSRC, f))
    out.append(os.path.join(INCLUDE, "rls_b200.h"))
    return out


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in _sources())


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    grid_o = os.path.join(BUILD, "grid.o")
    eng_o = os.path.join(BUILD, "engine.o")
    ic_o = os.path.join(BUILD, "icfact.o")
    mtx_o = os.path.join(BUILD, "mtxio.o")
    for src, obj in (("grid.cpp", grid_o), ("icfact.cpp", ic_o), ("mtxio.cpp", mtx_o)):
        _run(["g++", "-std=c++17", "-O2", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-c",
              os.path.join(CSRC, src), "-o", obj])
    cmd = [NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-c",
           os.path.join(CSRC, "engine.cu"), "-o", eng_o]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    _run(cmd)
    tmp = LIB + ".tmp"
    _run([NVCC, *ARCH, "-shared", "-o", tmp, eng_o, grid_o, ic_o, mtx_o, "-lcudart", "-lpthread"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="--ptxas" in sys.argv)
