"""Build the codec library in-tree: cuda_bpc-paco_b200/libbpc_paco.so.

    python cuda_bpc-paco_b200/build.py [--force]

nvcc compiles the sm_100a kernels and the C ABI into one shared library
(static CUDA runtime, so the library loads with or without torch in the
process).  No GPU is needed to build.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libbpc_paco.so")
SOURCES = ["bpc_kernels.cu", "bpc_order.cu", "bpc_api.cu", "bpc_batch.cu", "bpc_noalloc.cu", "bpc_dwt.cu", "bpc_server.cu",
           "bpc_train.cu", "bpc_lut.cpp", "bpc_files.cpp"]
HEADERS = ["bpc_core.cuh", "bpc_kernels.h", "bpc_lut.h", "bpc_arena.h"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "-shared", "-Xptxas", "-O3"]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS] + [os.path.join(ROOT, "include", "bpc_paco.h"),
                                                                os.path.abspath(__file__)]
    if force or _stale(LIB, deps):
        cmd = [NVCC, *ARCH, *FLAGS, "-I", os.path.join(ROOT, "include"), "-o", LIB + ".tmp",
               *[os.path.join(CSRC, f) for f in SOURCES]]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
