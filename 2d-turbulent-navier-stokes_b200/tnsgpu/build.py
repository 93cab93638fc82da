"""In-tree build of libtnsgpu.so for sm_100a (nvcc, no JIT cache)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "csrc")
SOURCES = ("tns_kernels.cu", "tns_kernels_mx.cu", "tns_api.cu", "tns_batch_api.cu", "tns_adjoint.cu",
           "tns_unstructured.cu", "tns_unstructured_mx.cu")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
# the mixed-precision kernels: FP32 division and square root to 2 ulp and FP32
# denormals flushed (their FP32 parts are deviations and sources whose error budget is
# FP32-level anyway; the FP64 parts are unaffected by these flags)
FILE_FLAGS = {"tns_kernels_mx.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"],
              "tns_unstructured_mx.cu": ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]}


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


def _obj_cmds(out: str, ti: int, verbose: bool):
    """One nvcc per source (with its own flags) into objects beside ``out``."""
    objs, cmds = [], []
    for src in SOURCES:
        obj = f"{out}.{os.path.splitext(src)[0]}.o"
        cmd = ["nvcc", *NVCC_FLAGS, *FILE_FLAGS.get(src, []), f"-DTNS_TI={ti}", "-c",
               os.path.join(CSRC, src), "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        objs.append(obj)
        cmds.append(cmd)
    return objs, cmds


def build_library(verbose: bool = False, variants: bool = True) -> str:
    """libtnsgpu.so (tile height TI = 8) and, with ``variants``, the TI = 4 and TI = 16
    builds the autotuner chooses among (compiled concurrently)."""
    from ._lib import TILE_VARIANTS
    jobs = [(TILE_VARIANTS[8], 8)]
    if variants:
        jobs += [(TILE_VARIANTS[t], t) for t in sorted(TILE_VARIANTS) if t != 8]
    plan = [(out, *_obj_cmds(out, ti, verbose)) for out, ti in jobs]
    procs = [(cmd[-1], subprocess.Popen(cmd)) for _, _, cmds in plan for cmd in cmds]
    failed = [obj for obj, p in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, f"nvcc for {failed}")
    for out, objs, _ in plan:
        subprocess.run(["nvcc", *ARCH, "-shared", *objs, "-o", out], check=True)
        for o in objs:
            os.remove(o)
    return TILE_VARIANTS[8]
