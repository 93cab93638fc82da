"""Fixed-point (steady-state) adjoint on a case that converges -- TEST INFRASTRUCTURE:
it checks the product's CUDA fixed-point adjoint against central finite differences of
the converged objective and prints the figures; run by hand on a GPU machine:

  python oracle/adjoint_steady_report.py [--nx 64] [--ny 24] [--cfl 0.5] [--tol 1e-6]
                                         [--adjoint-iters 600000] [--fd-iters 700000]
                                         [--max-primal 2000000]

The compression ramp (BCs as the 192 x 64 ramp case) at NX x NY cells and CFL 0.5, the
one configuration of the ramp family whose explicit iteration converges.
1. The primal runs on the GPU (FP64) from the cold start in blocks of 10 000 iterations
   until max_k CDIFF_k / CDIFF_k(first block) < tol.
2. The fixed-point adjoint of the wall pressure force J = F_y at that state: frozen
   CUDA adjoint steps lambda <- dJ/dQ + lambda dG/dQ (tns_adjoint_step), then the
   steady gradient dJ/dp = dJ/dp|direct + lambda dG/dp for P0, T0 and the y of ramp-wall
   node i = 3/4 NX, blended to zero at the top.
3. Central finite differences of the steady J for P0 and the wall node: the primal is
   warm-started from the converged state at p +- h (relative step 1e-6, node 3e-7 m)
   and run ``--fd-iters`` iterations, enough for the perturbation to settle (the
   iteration contracts by about 0.85 per 10 000 iterations here).

Prints one JSON object.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "2d-turbulent-navier-stokes_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def converge(Solver, mesh, flow, rinit, c0, tol, max_iter, first=None):
    """Runs the GPU primal from c0 until the residual ratio drops below tol; returns
    (state, iterations, ratio, first-block CDIFF)."""
    s = Solver(mesh, flow, rinit, precision=0)
    try:
        s.upload(c0)
        n, ratio = 0, float("inf")
        while n < max_iter:
            rec = s.run(10000, 10000)
            n += 10000
            if first is None:
                first = rec[0]
            ratio = float(np.max(rec[-1] / first))
            if ratio < tol:
                break
        return s.download(), n, ratio, first
    finally:
        s.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--ny", type=int, default=24)
    ap.add_argument("--cfl", type=float, default=0.5)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--adjoint-iters", type=int, default=600000)
    ap.add_argument("--fd-iters", type=int, default=700000)
    ap.add_argument("--max-primal", type=int, default=2000000)
    a = ap.parse_args()
    import torch
    from tnsgpu import adjoint, cases, formats
    from tnsgpu.solver import Solver
    nx, ny = a.nx, a.ny
    mesh = cases.ramp_mesh(nx, ny)
    flow = formats.Flow(**{**cases.ramp_flow().__dict__, "cfl": a.cfl})
    flow.istart = 0
    node = (3 * nx) // 4
    sch = adjoint.Scheme(mesh, flow, device="cuda")
    blend = 1.0 - cases.stretch_one_sided(ny, cases.beta_for_first_cell(ny, 0.3, 1e-5))
    space = adjoint.DesignSpace(sch, adjoint.ramp_wall_shape(sch, [node], blend))
    out = {"case": f"ramp_{nx}x{ny}_cfl{a.cfl}", "objective": "wall_force_y", "wall_node": node}
    prm = sch.params()
    rinit = float(sch.rtol(prm) / flow.rtred)
    c0 = sch.cold_state(prm).reshape(5, -1).cpu().numpy()
    t0 = time.perf_counter()
    q, n, ratio, first = converge(Solver, mesh, flow, rinit, c0, a.tol, a.max_primal)
    out["primal"] = {"iterations": n, "residual_ratio": ratio, "seconds": time.perf_counter() - t0}
    print(json.dumps({"primal": out["primal"]}), file=sys.stderr, flush=True)
    qstar = torch.tensor(q.reshape(5, nx, ny), device="cuda")
    dy = torch.zeros(1, dtype=torch.float64)
    t0 = time.perf_counter()
    fp = adjoint.fixed_point_adjoint(sch, adjoint.wall_force_y, qstar, niter=a.adjoint_iters, dy=dy, space=space,
                                     history_every=50000)
    torch.cuda.synchronize()
    out["fixed_point"] = {"iterations": a.adjoint_iters, "seconds": time.perf_counter() - t0,
                          "residual_every_50k": fp["residual_history"]}
    print(json.dumps({"fixed_point": out["fixed_point"], "grads": {"p0": fp["dJ_dp0"], "dy": float(fp["dJ_ddy"][0])}}),
          file=sys.stderr, flush=True)
    grads = {"p0": fp["dJ_dp0"], "t0": fp["dJ_dt0"], "dy": float(fp["dJ_ddy"][0])}

    def J_at(which, value):
        f, m = flow, mesh
        if which == "p0":
            f = dataclasses.replace(flow, p0=value)
        elif which == "t0":
            f = dataclasses.replace(flow, t0=value)
        d = torch.tensor([value if which == "dy" else 0.0], dtype=torch.float64, device="cuda")
        if which == "dy":
            m = adjoint._mesh_with_coords(sch, space, d)
        p = sch.params(f.p0, f.t0)
        s = Solver(m, f, float(sch.rtol(p) / flow.rtred), precision=0)
        try:
            s.upload(q)
            s.run(a.fd_iters, 0)
            qq = s.download()
        finally:
            s.close()
        x, y = space.coords(d.to("cuda"))
        C = torch.tensor(qq.reshape(5, nx, ny), device="cuda")
        return float(adjoint.wall_force_y(sch, C, sch.geometry(x, y), p))

    fd = {}
    t0 = time.perf_counter()
    for which, base, h in (("p0", flow.p0, 1e-6 * flow.p0), ("dy", 0.0, 3e-7)):
        v = (J_at(which, base + h) - J_at(which, base - h)) / (2 * h)
        fd[which] = {"adjoint": grads[which], "fd": v, "rel_diff": abs(grads[which] - v) / max(abs(v), 1e-300)}
        print(json.dumps({which: fd[which]}), file=sys.stderr, flush=True)
    fd["t0"] = {"adjoint": grads["t0"]}
    out["finite_differences"] = fd
    out["fd_seconds"] = time.perf_counter() - t0
    print(json.dumps(out))


if __name__ == "__main__":
    main()
