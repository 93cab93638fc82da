"""In-tree build of libtnsgpu.so for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "csrc")
SOURCES = ("tns_kernels.cu", "tns_api.cu")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


def build_library(verbose: bool = False) -> str:
    out = os.path.join(HERE, "libtnsgpu.so")
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = ["nvcc", *NVCC_FLAGS, *srcs, "-o", out]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    return out
