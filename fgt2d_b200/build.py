"""Builds the in-tree shared library ``fgt2d_b200/lib/libfgt_b200.so``.

nvcc compiles the CUDA stages for sm_100a only and the host tree/plan/C-ABI
sources with the system g++ (OpenMP).  The library has no PyTorch dependency:
it is the drop-in binary a Fortran, C or Python caller links or loads.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libfgt_b200.so")
SOURCES = ["fgt_kernels.cu", "fgt_devtree.cu", "fgt_tree.cpp", "fgt_plan.cpp", "fgt_capi.cpp"]
HEADERS = ["fgt_tree.hpp", "fgt_plan.hpp", "fgt_device.hpp"]
ARCH = "-gencode=arch=compute_100a,code=sm_100a"


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build fgt2d_b200")


def _ccbin() -> list[str]:
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return ["-ccbin", cand]
    return []


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "fgt_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *_ccbin(), "-O3", "-std=c++17", ARCH, "-lineinfo", "-shared",
           "-Xcompiler", "-fPIC,-fopenmp,-O3", "-Xptxas", "-O3",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
           *[os.path.join(CSRC, f) for f in SOURCES], "-o", tmp, "-lgomp", "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
