"""Generates tests/golden/case1.npz from the reference's own example case.

The reference ships one runnable case, examples/case1 (flow.in, grid.in, bc.in; its
README.md:16-24 runs it): a 115 x 50 cell 2-D channel with BC types 2, 3, 4 and 5, cold
start (ISTART=0), IAXIS=0, LOCAL=1.  It has no outputs, so this script stores:

* the case's inputs exactly as the reference's reader sees them (grid.in millimetre
  coordinates, NOD / NC connectivity, the bc.in columns, the 17 flow.in values), so that
  the GPU tests can run the case on a machine without the reference tree;
* the oracle's state and CDIFF history after NITER iterations from the cold start
  (monitor every MONITOR iterations).

Run in a tree where the reference is mounted:  python tests/golden/make_case1.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "2d-turbulent-navier-stokes_b200"))

from oracle.pyoracle import Oracle  # noqa: E402
from tnsgpu import formats  # noqa: E402

CASE_DIR = "/root/reference/examples/case1"
NITER, MONITOR = 1000, 100
FLOW_KEYS = ("gama", "amol", "local", "niter", "istart", "cfl", "prandtl", "prandtlt", "p0",
             "t0", "pamb", "amachinit", "rtred", "npseudo", "iaxis")


def read_reference_case(case_dir: str = CASE_DIR):
    """(Mesh, Flow) of the case files, through the same readers the drop-in main mirrors."""
    flow = formats.read_flow(os.path.join(case_dir, "flow.in"))
    mesh = formats.read_grid_bc(os.path.join(case_dir, flow.fnamegrid),
                                os.path.join(case_dir, flow.fnamebc))
    return mesh, flow


def main():
    mesh, flow = read_reference_case()
    ri = formats.rinit_cold(flow)
    o = Oracle(mesh, flow, ri)
    o.cold_start()
    hist = o.iterate(NITER, MONITOR)
    np.savez_compressed(
        os.path.join(HERE, "case1.npz"),
        x_mm=mesh.x_mm, y_mm=mesh.y_mm, nod=mesh.nod, nc=mesh.nc,
        bc=np.stack([mesh.nparent, mesh.nghost, mesh.ntype, mesh.nside], axis=1),
        flow=np.array([float(getattr(flow, k)) for k in FLOW_KEYS]),
        state=o.state(), cdiff=hist,
        rinit=ri, niter=NITER, monitor=MONITOR)
    print("case1", mesh.neles, "cells,", NITER, "iterations, final CDIFF", hist[-1])


if __name__ == "__main__":
    main()
