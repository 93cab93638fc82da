"""In-tree build of libtnsgpu.so for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "csrc")
SOURCES = ("tns_kernels.cu", "tns_kernels_mx.cu", "tns_api.cu", "tns_batch_api.cu")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared"]


MAINS = os.path.join(os.path.dirname(HERE), "mains")


def build_mains() -> list:
    """twodturb / axiturb: the main program with the RK4 loop on the GPU (g++, linked
    against the in-tree libtnsgpu.so).  Both read IAXIS from flow.in; they differ only
    in the default used when flow.in has 16 values."""
    out = []
    for name, iaxis in (("twodturb", 0), ("axiturb", 1)):
        exe = os.path.join(MAINS, name)
        subprocess.run(["g++", "-O2", "-std=c++17", f"-DTNS_DEFAULT_IAXIS={iaxis}",
                        os.path.join(MAINS, "tnsmain.cpp"), "-o", exe, f"-L{HERE}", "-ltnsgpu",
                        "-Wl,-rpath,$ORIGIN/../tnsgpu"], check=True)
        out.append(exe)
    return out


def _lib_cmd(out: str, ti: int, verbose: bool):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    cmd = ["nvcc", *NVCC_FLAGS, f"-DTNS_TI={ti}", *srcs, "-o", out]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    return cmd


def build_library(verbose: bool = False, variants: bool = True) -> str:
    """libtnsgpu.so (tile height TI = 8) and, with ``variants``, the TI = 4 and TI = 16
    builds the autotuner chooses among (compiled concurrently)."""
    from ._lib import TILE_VARIANTS
    jobs = [(TILE_VARIANTS[8], 8)]
    if variants:
        jobs += [(TILE_VARIANTS[t], t) for t in sorted(TILE_VARIANTS) if t != 8]
    procs = [(out, subprocess.Popen(_lib_cmd(out, ti, verbose))) for out, ti in jobs]
    failed = [out for out, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, f"nvcc for {failed}")
    return TILE_VARIANTS[8]
