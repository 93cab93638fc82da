"""Batched parameter sweep against the same cases solved one after another.

Builds the seeded ramp sweep (``cases.ramp_sweep``: 64 cases, 96x32 .. 512x192 cells,
ramp angle, P0 and T0 drawn per case), cold-starts every case and runs it, in the
mixed FP32/FP64 mode, until its residual ratio max_k CDIFF_k / CDIFF_k(iteration 1)
reaches ``stop_ratio`` at a record (every ``monitor`` iterations) or ``niter``
iterations pass -- once as one batch (tns_batch_run: every kernel phase is one launch
over the tiles of all active cases, converged cases masked off) and once case by case
through tns_run with the same criterion.  Reports both wall times (device work
synchronised, state uploads excluded), the iterations each case ran, and whether
every batched final state equals its sequential counterpart bit for bit.

  python -m tnsgpu.sweep [--cases 64] [--niter 5000] [--stop-ratio 1e-5] [--monitor 1000]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases, formats
from .batch import Batch
from .solver import Solver


def _solvers(sweep, precision):
    out = []
    for c in sweep:
        mesh, flow = c.mesh(), c.flow()
        ri = formats.rinit_cold(flow)
        s = Solver(mesh, flow, ri, precision=precision)
        s.upload(formats.cold_state(flow, mesh.neles, ri))
        out.append(s)
    return out


def run_sequential(solvers, niter, monitor, stop_ratio):
    """Each case alone: iteration 1 monitored (the reference), then chunks ending on the
    monitor cadence, stopping at the criterion -- the batch's schedule, case by case."""
    iters = []
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


def run_batched(solvers, niter, monitor, stop_ratio):
    b = Batch(solvers)
    t0 = time.perf_counter()
    r = b.run(niter, monitor, stop_ratio)
    dt = time.perf_counter() - t0
    launches = b.launch_count()
    b.close()
    return dt, [int(v) for v in r.iterations], launches


def compare(ncases=64, niter=5000, stop_ratio=1.0e-5, monitor=1000, seed=0, precision=1):
    sweep = cases.ramp_sweep(ncases, seed=seed)
    cells = np.array([c.nx * c.ny for c in sweep])
    # warm-up: library load, kernel attributes, a graph capture on a small batch
    warm = _solvers(sweep[:2], precision)
    run_batched(warm, 3, 0, 0.0)
    for s in warm:
        s.run(2, 0)
        s.close()

    seq = _solvers(sweep, precision)
    t_seq, it_seq = run_sequential(seq, niter, monitor, stop_ratio)
    q_seq = [s.download() for s in seq]
    for s in seq:
        s.close()

    bat = _solvers(sweep, precision)
    t_bat, it_bat, launches = run_batched(bat, niter, monitor, stop_ratio)
    same = [bool(np.array_equal(s.download(), q)) for s, q in zip(bat, q_seq)]
    for s in bat:
        s.close()
    work = float(np.sum(cells * np.array(it_bat)))
    return {
        "cases": ncases, "seed": seed, "precision": "mixed" if precision else "fp64",
        "cells_total": int(cells.sum()), "niter": niter, "monitor": monitor, "stop_ratio": stop_ratio,
        "batched_s": t_bat, "sequential_s": t_seq, "speedup": t_seq / t_bat,
        "batched_cell_iter_per_s": work / t_bat, "sequential_cell_iter_per_s": work / t_seq,
        "iterations_equal": it_bat == it_seq, "states_bitwise_equal": all(same),
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
    a = ap.parse_args()
    print(json.dumps(compare(a.cases, a.niter, a.stop_ratio, a.monitor, a.seed,
                             1 if a.precision == "mixed" else 0)))


if __name__ == "__main__":
    main()
