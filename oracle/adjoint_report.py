"""Full-size adjoint check on the 512 x 192 ramp -- TEST INFRASTRUCTURE: it checks the
product's CUDA adjoint against central finite differences of the GPU FP64 path and of
the oracle, and prints the figures; run by hand on a GPU machine:

  python oracle/adjoint_report.py [--primal-iters 5000] [--transient-iters 500]
                                  [--fixed-point-iters 200] [--oracle-fd]

Geometry and BCs as the 192 x 64 ramp case, at 512 x 192 cells.  Parameters: P0, T0,
AMACHINIT and the displacements of the 64 ramp-wall nodes i = 260, 264, ..., 512 (every
4th of the ramp's 257 wall nodes), evaluated at a seeded N(0, 1e-4 m) displacement
(numpy default_rng(0)), each blended linearly to zero at the top boundary.

1. A ``--primal-iters`` GPU FP64 run from the cold start, reporting the residual ratio
   (CDIFF at the end over CDIFF of iteration 1), then the fixed-point adjoint at that
   state (adjoint residual history).
2. The transient gradient of J(Q_N), N = ``--transient-iters``, from the cold start:
   primal on the GPU through the C ABI with a checkpoint (or a record of the forward
   values) per iteration, reverse sweep of CUDA adjoint steps (tnsgpu.adjoint).  Two objectives: the wall pressure force (y) and the
   total-pressure loss between the inlet (side 4) and the outlet (side 2).
3. Central finite differences of both objectives for 4 parameters -- P0, T0, AMACHINIT
   and wall node i = 388 -- on the GPU FP64 path, and with ``--oracle-fd`` on the
   oracle (C, host cores, one process per evaluation), at steps h and 3h with the
   Richardson value D(h) + (D(h) - D(3h)) / 8.  h is relative 1e-3 for P0 and
   AMACHINIT, 1e-2 for T0 (J is nearly independent of T0, so a smaller step returns
   rounding noise) and 3e-7 m for the node.
4. With ``--step-study``: the GPU central differences of T0, P0 and AMACHINIT over
   relative steps 3e-2 .. 1e-7, and of the node over 1e-8 .. 1e-4 m.

Prints one JSON object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import dataclasses
import json
import multiprocessing as mp
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "2d-turbulent-navier-stokes_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

NX, NY = 512, 192
WALL = list(range(260, 513, 4))
CHECK_NODE = WALL.index(388)


def _setup(device):
    import torch
    from tnsgpu import adjoint, cases
    mesh, flow = cases.ramp_mesh(NX, NY), cases.ramp_flow()
    flow.istart = 0
    sch = adjoint.Scheme(mesh, flow, device=device)
    blend = 1.0 - cases.stretch_one_sided(NY, cases.beta_for_first_cell(NY, 0.3, 1e-5))
    space = adjoint.DesignSpace(sch, adjoint.ramp_wall_shape(sch, WALL, blend))
    dy = torch.tensor(np.random.default_rng(0).normal(0.0, 1e-4, len(WALL)), dtype=torch.float64)
    return mesh, flow, sch, space, dy


def _oracle_objective(args):
    """One oracle evaluation (runs in a child process)."""
    which, value, niter, objective = args
    import torch
    from oracle.pyoracle import Oracle
    from tnsgpu import adjoint
    mesh, flow, sch, space, dy = _setup("cpu")
    kw = {"p0": flow.p0, "t0": flow.t0, "am": flow.amachinit}
    if which in kw:
        kw[which] = value
    else:
        dy = dy.clone()
        dy[CHECK_NODE] = value
    prm = sch.params(kw["p0"], kw["t0"], kw["am"])
    c0 = sch.cold_state(prm).reshape(5, -1).numpy()
    x, y = space.coords(dy)
    m = dataclasses.replace(mesh, x=x.numpy().ravel().copy(), y=y.numpy().ravel().copy())
    f = dataclasses.replace(flow, p0=kw["p0"], t0=kw["t0"], amachinit=kw["am"])
    o = Oracle(m, f, float(sch.rtol(prm) / flow.rtred))
    o.set_state(c0)
    o.iterate(niter, 0)
    C = torch.tensor(o.state().reshape(5, NX, NY))
    return float(getattr(adjoint, objective)(sch, C, sch.geometry(x, y), prm))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--primal-iters", type=int, default=5000)
    ap.add_argument("--transient-iters", type=int, default=500)
    ap.add_argument("--fixed-point-iters", type=int, default=200)
    ap.add_argument("--oracle-fd", action="store_true")
    ap.add_argument("--step-study", action="store_true")
    a = ap.parse_args()
    # the oracle pool starts before any CUDA work
    pool = cf.ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1),
                                  mp_context=mp.get_context("spawn")) if a.oracle_fd else None
    import torch
    from tnsgpu import adjoint
    from tnsgpu.solver import Solver
    mesh, flow, sch, space, dy = _setup("cuda")
    out = {"case": f"ramp_{NX}x{NY}", "parameters": 3 + len(WALL), "check_node": WALL[CHECK_NODE]}
    prm = sch.params()
    objectives = ("wall_force_y", "total_pressure_loss")

    # 1. long primal + fixed-point adjoint at its final state
    with torch.no_grad():
        c0 = sch.cold_state(prm).reshape(5, -1).cpu().numpy()
        m = adjoint._mesh_with_coords(sch, space, dy.to(sch.device))
    s = Solver(m, flow, float(sch.rtol(prm) / flow.rtred), precision=0)
    s.upload(c0)
    first = s.run(1, 1)[0]
    t0 = time.perf_counter()
    rec = s.run(a.primal_iters - 1, 1000)
    out["primal"] = {"iterations": a.primal_iters, "seconds": time.perf_counter() - t0,
                     "residual_ratio": float(np.max(rec[-1] / first)) if len(rec) else None}
    qstar = torch.tensor(s.download().reshape(5, NX, NY), device=sch.device)
    s.close()
    t0 = time.perf_counter()
    fp = adjoint.fixed_point_adjoint(sch, adjoint.wall_force_y, qstar, niter=a.fixed_point_iters,
                                     dy=dy.to(sch.device), space=space)
    h = fp["residual_history"]
    out["fixed_point"] = {"iterations": len(h), "seconds": time.perf_counter() - t0,
                          "adjoint_residual_first_last": [h[0], h[-1]] if h else None,
                          "dJ_dp0": fp["dJ_dp0"]}
    del fp, qstar
    torch.cuda.empty_cache()

    # 2. transient gradients
    N = a.transient_iters
    grads = {}
    for obj in objectives:
        t0 = time.perf_counter()
        r = adjoint.transient_gradient(sch, getattr(adjoint, obj), dy=dy.to(sch.device), space=space,
                                       niter=N)
        total = time.perf_counter() - t0
        grads[obj] = r
        out[obj] = {"J": r["J"], "dJ_dp0": r["dJ_dp0"], "dJ_dt0": r["dJ_dt0"],
                    "dJ_damachinit": r["dJ_damachinit"], "dJ_ddy_check_node": float(r["dJ_ddy"][CHECK_NODE]),
                    "dJ_ddy_norm": float(np.linalg.norm(r["dJ_ddy"])), "seconds_total": total}
        del r["states"]
    # primal alone at this size, for the adjoint / primal time ratio
    s = Solver(m, flow, float(sch.rtol(prm) / flow.rtred), precision=0)
    s.upload(c0)
    s.run(5, 0)
    t0 = time.perf_counter()
    s.run(N, 0)
    out["primal_seconds_transient_iters"] = time.perf_counter() - t0
    s.close()

    # 3. finite differences on the GPU FP64 path (and the oracle)
    base = {"p0": flow.p0, "t0": flow.t0, "am": flow.amachinit, "dy": float(dy[CHECK_NODE])}
    steps = {"p0": 1e-3 * flow.p0, "t0": 1e-2 * flow.t0, "am": 1e-3 * flow.amachinit, "dy": 3e-7}

    def gpu_J(obj, which, value):
        kw = {"p0": None, "t0": None, "amachinit": None, "dy": dy}
        if which == "dy":
            d = dy.clone()
            d[CHECK_NODE] = value
            kw["dy"] = d
        else:
            kw[{"p0": "p0", "t0": "t0", "am": "amachinit"}[which]] = value
        return adjoint.objective_gpu(sch, getattr(adjoint, obj), kw["p0"], kw["t0"], kw["amachinit"],
                                     kw["dy"], space, N)

    key = {"p0": "dJ_dp0", "t0": "dJ_dt0", "am": "dJ_damachinit"}
    fd = {}
    jobs = []
    for obj in objectives:
        for which in base:
            adj = grads[obj]["dJ_ddy"][CHECK_NODE] if which == "dy" else grads[obj][key[which]]
            row = {"adjoint": float(adj)}
            for mult in (1, 3):
                hh = mult * steps[which]
                row[f"gpu_fd_h{mult}"] = (gpu_J(obj, which, base[which] + hh) -
                                          gpu_J(obj, which, base[which] - hh)) / (2 * hh)
                if pool is not None:
                    for sgn in (1, -1):
                        jobs.append(((obj, which, mult, sgn),
                                     pool.submit(_oracle_objective, (which, base[which] + sgn * hh, N, obj))))
            row["gpu_richardson"] = row["gpu_fd_h1"] + (row["gpu_fd_h1"] - row["gpu_fd_h3"]) / 8.0
            row["rel_diff_gpu_fd"] = abs(row["adjoint"] - row["gpu_fd_h1"]) / max(abs(row["gpu_fd_h1"]), 1e-300)
            row["rel_diff_gpu_richardson"] = abs(row["adjoint"] - row["gpu_richardson"]) / \
                max(abs(row["gpu_richardson"]), 1e-300)
            fd[f"{obj}/{which}"] = row
    if pool is not None:
        vals = {k: f.result() for k, f in jobs}
        for obj in objectives:
            for which in base:
                row = fd[f"{obj}/{which}"]
                for mult in (1, 3):
                    hh = mult * steps[which]
                    row[f"oracle_fd_h{mult}"] = (vals[(obj, which, mult, 1)] - vals[(obj, which, mult, -1)]) / (2 * hh)
                row["rel_diff_oracle_fd"] = abs(row["adjoint"] - row["oracle_fd_h1"]) / \
                    max(abs(row["oracle_fd_h1"]), 1e-300)
        pool.shutdown()
    out["finite_differences"] = fd
    if a.step_study:
        study = {}
        for obj in objectives:
            for which in base:
                adj = grads[obj]["dJ_ddy"][CHECK_NODE] if which == "dy" else grads[obj][key[which]]
                rels = (1e-8, 3e-8, 1e-7, 3e-7, 1e-6, 3e-6, 1e-5, 3e-5, 1e-4) if which == "dy" else \
                    (3e-2, 1e-2, 3e-3, 1e-3, 3e-4, 1e-4, 3e-5, 1e-5, 3e-6, 1e-6, 3e-7, 1e-7)
                rows = []
                for rel in rels:
                    hh = rel if which == "dy" else rel * base[which]
                    c = (gpu_J(obj, which, base[which] + hh) - gpu_J(obj, which, base[which] - hh)) / (2 * hh)
                    rows.append({"step": rel, "central": c,
                                 "rel_diff": abs(float(adj) - c) / max(abs(c), 1e-300)})
                study[f"{obj}/{which}"] = {"adjoint": float(adj), "rows": rows}
        out["step_study"] = study
    print(json.dumps(out))


if __name__ == "__main__":
    main()
