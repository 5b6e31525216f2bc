"""Build libctlab_b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python ct_laboratory_b200/build.py [--force]   # (not -m: that would import the package,
                                                   #  which needs the library already built)

The library lands in ct_laboratory_b200/_lib/ next to the package so that it
travels with the source tree; the loader (ct_laboratory_b200/_native.py)
refuses to run without it.  nvcc cross-compiles, so no GPU is needed here.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIB_DIR, "libctlab_b200.so")
INCLUDE = os.path.join(ROOT, "include")

SOURCES = ["capi.cu", "siddon.cu", "tvals.cu", "gather.cu", "batched.cu", "map_step.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: set NVCC or put the CUDA toolkit on PATH")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra=None) -> str:
    """Compile every .cu source into one shared library; returns its path."""
    if not force and not _stale():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O2",
           "-Xptxas", "-warn-spills", "-I", INCLUDE, "-I", CSRC, "-o", tmp,
           *[os.path.join(CSRC, s) for s in SOURCES], *(extra or [])]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    # nvcc picks the host compiler from CC/CXX-independent defaults; the image
    # exports CC=/opt/gcc/bin/gcc, which is fine for C++ host code.
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose and (res.stdout or res.stderr):
        print(res.stdout + res.stderr, file=sys.stderr)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
