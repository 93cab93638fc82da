"""Golden fixtures (tests/golden/make_golden.py): the oracle must keep reproducing them
(CPU), and the CUDA path must match them to the parity tolerance (GPU)."""
import os

import numpy as np
import pytest

from oracle.pyoracle import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))
NAMES = ["ramp_24x10", "nozzle2d_20x12", "port_axi_20x10", "ramp_global_dt_16x8"]


def _load(name):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    from make_golden import golden_cases
    m, f, c0, ri, n, mon = golden_cases()[name]
    g = np.load(os.path.join(HERE, "golden", name + ".npz"))
    assert np.array_equal(g["c0"], c0) and float(g["rinit"]) == ri
    return m, f, c0, ri, int(g["niter"]), int(g["monitor"]), g


def _rel(a, b):
    return np.max(np.abs(a - b), axis=-1) / np.max(np.abs(b), axis=-1)


@pytest.mark.parametrize("name", NAMES)
def test_oracle_reproduces_golden(name):
    m, f, c0, ri, n, mon, g = _load(name)
    o = Oracle(m, f, ri)
    o.set_state(c0)
    hist = o.iterate(n, mon)
    assert np.all(_rel(o.state(), g["state"]) <= 1e-14)
    assert np.max(np.abs(hist - g["cdiff"]) / np.abs(g["cdiff"])) <= 1e-14


@pytest.mark.gpu
@pytest.mark.parametrize("name", NAMES)
def test_gpu_matches_golden(name):
    from tnsgpu.solver import Solver
    m, f, c0, ri, n, mon, g = _load(name)
    s = Solver(m, f, ri)
    s.upload(c0)
    hist = s.run(n, mon)
    assert np.all(_rel(s.download(), g["state"]) <= 1e-10)
    assert np.max(np.abs(hist - g["cdiff"]) / np.abs(g["cdiff"])) <= 1e-10
