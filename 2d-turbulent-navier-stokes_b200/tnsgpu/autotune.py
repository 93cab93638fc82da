"""Autotuner: tile height and batch schedule, chosen by timing the actual workload.

The tile kernels are compiled for three tile heights -- TI = 4, 8 or 16 rows of 32
cells per thread block (``libtnsgpu_ti4.so``, ``libtnsgpu.so``, ``libtnsgpu_ti16.so``;
each build keeps the threads resident per SM of the TI = 8 tuning).  A batch can also
run any of four schedules (0: one launch per kernel phase over the tiles of all cases;
1: the cases' own launches on parallel branches of one CUDA graph; 2: as 1 with 8
iterations per graph; 3: one persistent cooperative launch per run of unmonitored
iterations, grid barriers between the phases -- refused, and skipped here, when a case
has LOCAL=0 or a type-6 port).  ``tune_batch`` and
``tune_case`` time a few iterations of the caller's cases under every combination and
return the fastest.

The FP64 path computes every cell with the same arithmetic whatever the tiling, so its
results are bit-identical across tile heights and schedules.  The mixed path's flux
residual is an FP32 sum of deviations from a per-tile FP64 reference flux (the first
cell of the tile), so its results depend on the tile height at FP32 rounding level, and
are identical across schedules.
"""
from __future__ import annotations

import json
import os
import time
from typing import Callable, Iterable, List, Optional, Sequence

from . import _lib
from .batch import Batch
from .solver import Solver

TILE_HEIGHTS = (4, 8, 16)


def available_tile_heights(heights: Iterable[int] = TILE_HEIGHTS) -> List[int]:
    return [t for t in heights if os.path.exists(_lib.variant_path(t))]


def _time_batch(solvers: Sequence[Solver], schedule: int, iters: int, warmup: int) -> float:
    b = Batch(solvers, schedule=schedule)
    try:
        b.run(warmup, 0)
        b.prepare()
        t0 = time.perf_counter()
        b.run(iters, 0)
        return (time.perf_counter() - t0) / iters
    finally:
        b.close()


def tune_batch(make_solvers: Callable[[str], List[Solver]], iters: int = 40, warmup: int = 16,
               tile_heights: Iterable[int] = TILE_HEIGHTS, schedules: Sequence[int] = (0, 1, 2, 3),
               cache: Optional[str] = None, key: Optional[str] = None) -> dict:
    """make_solvers(lib_path) builds the batch's cases (state uploaded) from that library
    build.  Times ``iters`` iterations after ``warmup`` untimed ones and
    Batch.prepare (every graph the schedule launches captured before the timing) for
    every (tile height, schedule) and returns {"ti", "schedule", "lib", "s_per_iter", "trials"}.  With ``cache`` (a
    JSON file) and ``key``, a stored choice is returned without timing."""
    if cache and key and os.path.exists(cache):
        with open(cache) as fh:
            stored = json.load(fh)
        if key in stored:
            return stored[key]
    trials = []
    for ti in available_tile_heights(tile_heights):
        path = _lib.variant_path(ti)
        solvers = make_solvers(path)
        try:
            for sch in schedules:
                try:
                    trials.append({"ti": ti, "schedule": sch,
                                   "s_per_iter": _time_batch(solvers, sch, iters, warmup)})
                except _lib.TnsError as e:  # a build whose kernels do not fit this GPU
                    trials.append({"ti": ti, "schedule": sch, "error": str(e)})
        finally:
            for s in solvers:
                s.close()
    ok = [t for t in trials if "s_per_iter" in t]
    if not ok:
        raise RuntimeError(f"no tile variant ran: {trials}")
    best = min(ok, key=lambda t: t["s_per_iter"])
    out = {"ti": best["ti"], "schedule": best["schedule"], "lib": _lib.variant_path(best["ti"]),
           "s_per_iter": best["s_per_iter"], "trials": trials}
    if cache and key:
        stored = {}
        if os.path.exists(cache):
            with open(cache) as fh:
                stored = json.load(fh)
        stored[key] = out
        with open(cache, "w") as fh:
            json.dump(stored, fh, indent=1)
    return out


def tune_case(make_solver: Callable[[str], Solver], iters: int = 50, warmup: int = 5,
              tile_heights: Iterable[int] = TILE_HEIGHTS) -> dict:
    """Tile height for one case run through tns_run: {"ti", "lib", "s_per_iter", "trials"}."""
    trials = []
    for ti in available_tile_heights(tile_heights):
        s = make_solver(_lib.variant_path(ti))
        try:
            s.run(warmup, 0)
            s.prepare()
            t0 = time.perf_counter()
            s.run(iters, 0)
            trials.append({"ti": ti, "s_per_iter": (time.perf_counter() - t0) / iters})
        except _lib.TnsError as e:
            trials.append({"ti": ti, "error": str(e)})
        finally:
            s.close()
    ok = [t for t in trials if "s_per_iter" in t]
    if not ok:
        raise RuntimeError(f"no tile variant ran: {trials}")
    best = min(ok, key=lambda t: t["s_per_iter"])
    return {"ti": best["ti"], "lib": _lib.variant_path(best["ti"]), "s_per_iter": best["s_per_iter"],
            "trials": trials}
