"""Build libdmrgx.so in-tree for sm_100a with nvcc.

    python -m dmrg_b200.build          # or build() from Python

The library is self-contained (static CUDA runtime) and is loaded with ctypes
by ``dmrg_b200.native``.  Objects go to dmrg_b200/_build/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libdmrgx.so")

SOURCES = ["qmeta.cpp", "ctx.cu", "gemm_f64.cu", "noalloc.cu", "split.cu", "tc_gemm.cu", "split_plan.cu", "eig.cu", "qtensor.cu", "adjoint.cu", "plain.cu", "dmrg.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # the system g++ links the shared C++ runtime (a static copy inside a
    # dlopen'ed library misbehaved under Python)
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".h")]
    headers.append(os.path.join(ROOT, "include", "dmrgx.h"))
    objs = []
    flags = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", host_cxx(),
             "-I", os.path.join(ROOT, "include")] + ARCH
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if not force and _newer(o, [s] + headers):
            continue
        cmd = [nvcc()] + flags + ["-c", s, "-o", o]
        if src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"] if verbose else []
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not _newer(LIB, objs):
        cmd = [nvcc(), "-shared", "-ccbin", host_cxx()] + ARCH + objs + ["-o", LIB, "-ldl"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
