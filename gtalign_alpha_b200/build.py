"""Build the in-tree CUDA library libgtb200.so for sm_100a with nvcc."""
from __future__ import annotations

import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libgtb200.so")
SOURCES = ["gtb_kernels.cu", "gtb_api.cu", "gtb_adjoint.cu", "gtb_noalloc.cu", "gtb_cluster.cu",
           "gtb_index.cpp", "gtb_frg3.cu", "gtb_reader.cpp"]
HEADERS = ["gtb_device.cuh", "gtb_kernels.cuh", "gtb_gonnet.h"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # every fused multiply-add in the kernels is written out explicitly
    "-fmad=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fno-fast-math",
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    deps.append(os.path.join(ROOT, "include", "gtb200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    for s in SOURCES:
        obj = os.path.join(objdir, os.path.splitext(s)[0] + ".o")
        cmd = [nvcc()] + NVCC_FLAGS + ["-I", os.path.join(ROOT, "include"), "-c",
                                       os.path.join(CSRC, s), "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        objs.append(obj)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + ["-lcudart", "-lz"]
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
