"""Builds libvlgpu.so (the CUDA hot path and its C ABI) in-tree for sm_100a.

    python -m vlasiator_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvlgpu.so")
SOURCES = ["acc_map.cu", "moments_geometry.cu", "adjust.cu", "translate.cu", "fill.cu", "capi.cu", "serve.cu", "noalloc.cu", "launch.cu", "halo.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17", "--shared",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-ccbin", "/usr/bin/g++", "-Xptxas", "-warn-spills"]


def build(verbose: bool = False, extra=()) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    newest = max(os.path.getmtime(p) for p in srcs + [os.path.join(CSRC, "vlgpu_common.cuh"),
                                                       os.path.join(CSRC, "geometry.cuh"),
                                                       os.path.join(CSRC, "batch_internal.cuh"),
                                                       os.path.join(CSRC, "fused_ppm.cuh"),
                                                       os.path.join(CSRC, "moments_record.cuh"),
                                                       os.path.join(HERE, "..", "include", "vlgpu.h")])
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest and not extra:
        return LIB
    cmd = [NVCC, *FLAGS, *extra, *srcs, "-o", LIB]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=tuple(sys.argv[1:]))
