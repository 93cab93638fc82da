"""Generates tests/golden/*.npz: oracle outputs on small seeded cases.

The reference (Fortran) cannot be compiled on these machines and ships no outputs, so
these vectors come from the C oracle (oracle/tns_oracle.c).  They pin the oracle
against regressions and give the GPU tests fixed targets; they do not pin the oracle
to the reference.  Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "2d-turbulent-navier-stokes_b200"))

from oracle.pyoracle import Oracle  # noqa: E402
from tnsgpu import cases, formats  # noqa: E402


def golden_cases():
    """name -> (mesh, flow, initial state, RINIT, iterations, monitor interval)."""
    out = {}
    m, f = cases.ramp_mesh(24, 10), cases.ramp_flow()
    c, ri = cases.noisy_restart_state(f, m.neles)
    out["ramp_24x10"] = (m, f, c, ri, 200, 50)
    m, f = cases.nozzle_2d_mesh(20, 12), cases.nozzle_2d_flow()
    ri = formats.rinit_cold(f)
    out["nozzle2d_20x12"] = (m, f, formats.cold_state(f, m.neles, ri), ri, 200, 50)
    m, f = cases.port_mesh(20, 10), cases.port_flow()
    m.ntype[(m.ntype == 5) & (m.nside == 1)] = 4  # type-4 axis: well conditioned
    ri = formats.rinit_cold(f)
    out["port_axi_20x10"] = (m, f, formats.cold_state(f, m.neles, ri), ri, 100, 25)
    m, f = cases.ramp_mesh(16, 8), formats.Flow(**{**cases.ramp_flow().__dict__, "local": 0})
    c, ri = cases.noisy_restart_state(f, m.neles, seed=3)
    out["ramp_global_dt_16x8"] = (m, f, c, ri, 100, 25)
    return out


def main():
    for name, (m, f, c0, ri, n, mon) in golden_cases().items():
        o = Oracle(m, f, ri)
        o.set_state(c0)
        hist = o.iterate(n, mon)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), c0=c0, state=o.state(),
                            cdiff=hist, rinit=ri, niter=n, monitor=mon)
        print(name, m.shape, n, "iterations")


if __name__ == "__main__":
    main()
