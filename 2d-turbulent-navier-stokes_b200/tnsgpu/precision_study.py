"""FP64 vs mixed FP32/FP64 on the same case and iteration count.

Runs a case three times on the GPU -- FP64, FP64 from a start state perturbed by 1e-15
(relative, seeded), and mixed FP32/FP64 -- for the same number of RK4 iterations, and
reports for the mixed run the relative differences to FP64 of the wall pressure, the
integrated wall pressure force and the outlet mass flow, next to the same differences
for the perturbed FP64 run.  The flows of these cases are unsteady or converge very
slowly, so the perturbed run measures how much any difference at round-off level grows
by itself; the mixed error is meaningful relative to that envelope.  It also reports
the residual monitor (CDIFF, turbnstwod.f90:148-163) each run ends at, relative to its
first iteration, and the throughput of both precisions.

  python -m tnsgpu.precision_study [--case nozzle_plume_1024x384] [--iters 20000]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import cases, formats, objectives
from .solver import Solver

CASES = {
    "nozzle_plume_1024x384": lambda: (cases.nozzle_plume_mesh(1024, 384), cases.nozzle_plume_flow()),
    "nozzle_plume_256x96": lambda: (cases.nozzle_plume_mesh(256, 96), cases.nozzle_plume_flow()),
    "ramp_192x64": lambda: (cases.ramp_mesh(192, 64), cases.ramp_flow()),
    "port_4096x1536": lambda: (cases.port_mesh(4096, 1536), cases.port_flow()),
    "port_1024x384": lambda: (cases.port_mesh(1024, 384), cases.port_flow()),
}
# the wall whose pressure and force are reported: BC type and side (the port channel's
# injecting wall is type 6; the other cases' upper wall is type 5)
WALL = {"port_4096x1536": (6, 3), "port_1024x384": (6, 3)}


def run(mesh, flow, c0, rinit, precision, iters, monitor=1000, wall=(5, 3)):
    s = Solver(mesh, flow, rinit, precision=precision)
    s.upload(c0)
    first = s.run(1, 1)[0]
    hist = []
    t = 0.0
    it = 1
    status = "ok"
    try:
        while it < iters:
            n = min(monitor, iters - it)
            t0 = time.perf_counter()
            rec = s.run(n, n)
            t += time.perf_counter() - t0
            it += n
            hist.append((it, float(np.max(rec[-1] / first))))
    except Exception as e:  # a run that blows up reports where
        status = f"failed after {it} iterations: {e}"
    out = dict(status=status, iterations=it, history=hist,
               cell_iter_per_s=mesh.neles * (it - 1) / t if t > 0 else None)
    if status == "ok":
        prims = s.primitives()
        out.update(state=s.download(),
                   wall_p=objectives.wall_pressure(mesh, prims, flow.amol, side=wall[1], wall_type=wall[0])[1],
                   force=objectives.wall_force(mesh, prims, flow.amol, flow.iaxis, side=wall[1],
                                               wall_type=wall[0]),
                   mdot=objectives.outlet_mass_flow(mesh, prims, flow.amol, flow.iaxis, side=2))
    s.close()
    return out


def _errors(a, b):
    return {
        "wall_pressure_rel_max": float(np.max(np.abs(a["wall_p"] - b["wall_p"]) / np.abs(b["wall_p"]))),
        "wall_force_rel": float(np.linalg.norm(a["force"] - b["force"]) / np.linalg.norm(b["force"])),
        "outlet_mass_flow_rel": float(abs(a["mdot"] - b["mdot"]) / max(abs(b["mdot"]), 1e-300)),
        "state_rel_max": [float(v) for v in np.max(np.abs(a["state"] - b["state"]), axis=1) /
                          np.max(np.abs(b["state"]), axis=1)],
    }


def compare(case="nozzle_plume_1024x384", iters=20000, seed=0):
    mesh, flow = CASES[case]()
    rinit = formats.rinit_cold(flow)
    c0 = formats.cold_state(flow, mesh.neles, rinit)
    c1 = c0 * (1.0 + 1e-15 * np.random.default_rng(seed).standard_normal(c0.shape))
    wall = WALL.get(case, (5, 3))
    f64 = run(mesh, flow, c0, rinit, 0, iters, wall=wall)
    f64p = run(mesh, flow, c1, rinit, 0, iters, wall=wall)
    mx = run(mesh, flow, c0, rinit, 1, iters, wall=wall)
    out = {"case": case, "cells": mesh.neles, "iterations": iters, "wall": {"type": wall[0], "side": wall[1]},
           "fp64": {k: f64[k] for k in ("status", "iterations", "cell_iter_per_s")},
           "mixed": {k: mx[k] for k in ("status", "iterations", "cell_iter_per_s")},
           "fp64_final_residual_ratio": f64["history"][-1][1] if f64["history"] else None,
           "mixed_final_residual_ratio": mx["history"][-1][1] if mx["history"] else None}
    if f64["status"] == "ok" and mx["status"] == "ok":
        out["mixed_vs_fp64"] = _errors(mx, f64)
        out["speedup"] = mx["cell_iter_per_s"] / f64["cell_iter_per_s"]
    if f64["status"] == "ok" and f64p["status"] == "ok":
        out["fp64_perturbed_vs_fp64"] = _errors(f64p, f64)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="nozzle_plume_1024x384", choices=sorted(CASES))
    ap.add_argument("--iters", type=int, default=20000)
    a = ap.parse_args()
    print(json.dumps(compare(a.case, a.iters)))


if __name__ == "__main__":
    main()
