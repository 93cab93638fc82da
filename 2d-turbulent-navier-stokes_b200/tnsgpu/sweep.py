"""Batched parameter sweep against the same cases solved one after another.

Builds the seeded ramp sweep (``cases.ramp_sweep``: 64 cases, 96x32 .. 512x192 cells,
ramp angle, P0 and T0 drawn per case), cold-starts every case and runs it, in the
mixed FP32/FP64 mode, until its residual ratio max_k CDIFF_k / CDIFF_k(iteration 1)
reaches ``stop_ratio`` at a record (every ``monitor`` iterations) or ``niter``
iterations pass -- once as one batch (tns_batch_run: every kernel phase is one launch
over the tiles of all active cases, converged cases masked off) and once case by case
through tns_run with the same criterion.  Before the batched run the autotuner picks
the tile height and the batch schedule by timing a few iterations of the sweep itself
(its time is reported apart); the sequential solves use the default build.  Reports
both wall times (device work synchronised, state uploads and graph capture excluded),
the iterations each
case ran, and how far every batched final state is from its sequential counterpart
(bit-identical in FP64; FP32 rounding of the per-tile reference flux in the mixed mode
when the tuned tile height differs from the default).

  python -m tnsgpu.sweep [--cases 64] [--niter 5000] [--stop-ratio 1e-5] [--monitor 1000]
                         [--precision mixed|fp64] [--no-tune] [--manifest batch.in]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import autotune, cases, formats
from .batch import Batch
from .solver import Solver


def _solvers(sweep, precision, lib=None):
    out = []
    for c in sweep:
        mesh, flow = c.mesh(), c.flow()
        ri = formats.rinit_cold(flow)
        s = Solver(mesh, flow, ri, precision=precision, lib=lib)
        s.upload(formats.cold_state(flow, mesh.neles, ri))
        out.append(s)
    return out


def run_sequential(solvers, niter, monitor, stop_ratio):
    """Each case alone: iteration 1 monitored (the reference), then chunks ending on the
    monitor cadence, stopping at the criterion -- the batch's schedule, case by case.
    Every case's graphs are captured before the timing (Solver.prepare)."""
    iters = []
    for s in solvers:
        s.prepare()
    t0 = time.perf_counter()
    for s in solvers:
        ref = s.run(1, 1)[0]
        it = 1
        while it < niter:
            n = min(monitor - it % monitor, niter - it)
            rec = s.run(n, n)  # the chunk's last iteration is monitored
            it += n
            if stop_ratio > 0 and it % monitor == 0 and np.max(rec[-1] / ref) <= stop_ratio:
                break
        iters.append(it)
    return time.perf_counter() - t0, iters


def run_batched(solvers, niter, monitor, stop_ratio, schedule=0):
    b = Batch(solvers, schedule=schedule)
    b.prepare()  # the schedule's graphs captured before the timing
    t0 = time.perf_counter()
    r = b.run(niter, monitor, stop_ratio)
    dt = time.perf_counter() - t0
    launches = b.launch_count()
    b.close()
    return dt, [int(v) for v in r.iterations], launches


def compare(ncases=64, niter=5000, stop_ratio=1.0e-5, monitor=1000, seed=0, precision=1, tune=True,
            manifest=None):
    """``manifest``: a batch manifest file (formats.read_manifest) instead of the seeded
    sweep."""
    if manifest:
        sweep = [cases.SweepCase(**row) for row in formats.read_manifest(manifest)]
        ncases = len(sweep)
    else:
        sweep = cases.ramp_sweep(ncases, seed=seed)
    cells = np.array([c.nx * c.ny for c in sweep])
    # warm-up: library load, kernel attributes, a graph capture on a small batch
    warm = _solvers(sweep[:2], precision)
    run_batched(warm, 3, 0, 0.0)
    for s in warm:
        s.run(2, 0)
        s.close()

    t0 = time.perf_counter()
    if tune:
        choice = autotune.tune_batch(lambda lib: _solvers(sweep, precision, lib))
    else:
        choice = {"ti": 8, "schedule": 0, "lib": None, "trials": []}
    t_tune = time.perf_counter() - t0

    seq = _solvers(sweep, precision)
    t_seq, it_seq = run_sequential(seq, niter, monitor, stop_ratio)
    q_seq = [s.download() for s in seq]
    for s in seq:
        s.close()

    bat = _solvers(sweep, precision, choice["lib"])
    t_bat, it_bat, launches = run_batched(bat, niter, monitor, stop_ratio, choice["schedule"])
    q_bat = [s.download() for s in bat]
    for s in bat:
        s.close()
    same = all(np.array_equal(a, b) for a, b in zip(q_bat, q_seq))
    rel = max(float(np.max(np.max(np.abs(a - b), axis=1) / np.max(np.abs(b), axis=1)))
              for a, b in zip(q_bat, q_seq))
    work = float(np.sum(cells * np.array(it_bat)))
    return {
        "cases": ncases, "seed": seed, "precision": "mixed" if precision else "fp64",
        "cells_total": int(cells.sum()), "niter": niter, "monitor": monitor, "stop_ratio": stop_ratio,
        "tuned": {"ti": choice["ti"], "schedule": choice["schedule"], "tuning_s": t_tune,
                  "trials": [{k: v for k, v in t.items()} for t in choice["trials"]]},
        "batched_s": t_bat, "sequential_s": t_seq, "speedup": t_seq / t_bat,
        "batched_cell_iter_per_s": work / t_bat, "sequential_cell_iter_per_s": work / t_seq,
        "iterations_equal": it_bat == it_seq, "states_bitwise_equal": same, "state_rel_diff_max": rel,
        "converged_cases": int(sum(i < niter for i in it_bat)),
        "iterations_min_max": [min(it_bat), max(it_bat)], "batch_launches": launches,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--niter", type=int, default=5000)
    ap.add_argument("--stop-ratio", type=float, default=1.0e-5)
    ap.add_argument("--monitor", type=int, default=1000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="mixed")
    ap.add_argument("--no-tune", action="store_true", help="default tile height and schedule 0")
    ap.add_argument("--manifest", help="batch manifest of ramp cases (name nx ny angle_deg p0 t0 amachinit)")
    a = ap.parse_args()
    print(json.dumps(compare(a.cases, a.niter, a.stop_ratio, a.monitor, a.seed,
                             1 if a.precision == "mixed" else 0, not a.no_tune, a.manifest)))


if __name__ == "__main__":
    main()
