"""Builds the in-tree shared library ``fgt2d_b200/lib/libfgt_b200.so``.

nvcc compiles the CUDA stages for sm_100a only and the host tree/plan/C-ABI
sources with the system g++ (OpenMP), one object per source file (in
parallel; only stale objects are rebuilt), then links them.  The library has no PyTorch dependency:
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
OBJDIR = os.path.join(LIBDIR, "obj")
SOURCES = ["fgt_kernels.cu", "fgt_mixed.cu", "fgt_tc.cu", "fgt_shard.cu", "fgt_devtree.cu", "fgt_tree.cpp", "fgt_plan.cpp", "fgt_capi.cpp"]
HEADERS = ["fgt_tree.hpp", "fgt_plan.hpp", "fgt_device.hpp", "fgt_kcommon.cuh", "fgt_tc.cuh", "fgt_shard.hpp"]
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


def _obj(src: str) -> str:
    return os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")


def _compile_cmd(src: str, out: str) -> list[str]:
    return [_nvcc(), *_ccbin(), "-O3", "-std=c++17", ARCH, "-lineinfo", "-c",
            "-Xcompiler", "-fPIC,-fopenmp,-O3", "-Xptxas", "-O3",
            "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
            os.path.join(CSRC, src), "-o", out]


def _stale_obj(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    deps = [os.path.join(CSRC, src)] + [os.path.join(CSRC, h) for h in HEADERS]
    deps.append(os.path.join(ROOT, "include", "fgt_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles each source to an object (in parallel, only the stale ones)
    and links the shared library."""
    todo = [s for s in SOURCES if force or _stale_obj(s)]
    if not todo and os.path.exists(LIB) and all(
            os.path.getmtime(_obj(s)) <= os.path.getmtime(LIB) for s in SOURCES):
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    procs = []
    for s in todo:
        cmd = _compile_cmd(s, _obj(s) + ".tmp")
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((s, subprocess.Popen(cmd)))
    failed = [s for s, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed on {failed}")
    for s, _ in procs:
        os.replace(_obj(s) + ".tmp", _obj(s))
    tmp = LIB + ".tmp"
    cmd = [_nvcc(), *_ccbin(), ARCH, "-shared", "-Xcompiler", "-fopenmp",
           *[_obj(s) for s in SOURCES], "-o", tmp, "-lgomp", "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
