"""The reference's own example case (examples/case1: README.md:16-24), a 115 x 50 cell
2-D channel, BC types 2 / 3 / 4 / 5, cold start, IAXIS=0, LOCAL=1.

Its inputs and the oracle's outputs after 1000 iterations live in tests/golden/case1.npz
(generated by tests/golden/make_case1.py from the reference's files).  The CPU tests pin
the fixture to the reference's files (where the reference tree is present) and the
oracle to the fixture; the GPU tests run the case through the C ABI and through the
drop-in main and hold Q and the CDIFF history to <= 1e-10 relative (max-norm per
variable) of the oracle.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tnsgpu import formats

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "case1.npz")
REF_CASE = "/root/reference/examples/case1"
FLOW_KEYS = ("gama", "amol", "local", "niter", "istart", "cfl", "prandtl", "prandtlt", "p0",
             "t0", "pamb", "amachinit", "rtred", "npseudo", "iaxis")
TOL = 1e-10


def load_case1():
    """(Mesh, Flow, fixture) from the committed fixture."""
    g = np.load(FIXTURE)
    bc = g["bc"]
    mesh = formats.Mesh(x=g["x_mm"] * formats.MM_TO_M, y=g["y_mm"] * formats.MM_TO_M,
                        nod=g["nod"].astype(np.int32), nc=g["nc"].astype(np.int32),
                        nparent=bc[:, 0].copy(), nghost=bc[:, 1].copy(),
                        ntype=bc[:, 2].copy(), nside=bc[:, 3].copy(),
                        x_mm=g["x_mm"], y_mm=g["y_mm"])
    flow = formats.Flow()
    for k, v in zip(FLOW_KEYS, g["flow"]):
        setattr(flow, k, type(getattr(flow, k))(v))
    return mesh, flow, g


def _rel(a, b):
    return np.max(np.abs(a - b), axis=-1) / np.max(np.abs(b), axis=-1)


@pytest.mark.skipif(not os.path.isdir(REF_CASE), reason="reference tree not mounted")
def test_fixture_is_the_reference_case():
    """The fixture holds exactly what the reference's reader takes from its files."""
    mesh, flow, _ = load_case1()
    rf = formats.read_flow(os.path.join(REF_CASE, "flow.in"))
    rm = formats.read_grid_bc(os.path.join(REF_CASE, "grid.in"), os.path.join(REF_CASE, "bc.in"))
    for k in FLOW_KEYS:
        assert getattr(flow, k) == getattr(rf, k), k
    for k in ("x_mm", "y_mm", "x", "y", "nod", "nc", "nparent", "nghost", "ntype", "nside"):
        assert np.array_equal(getattr(mesh, k), getattr(rm, k)), k


def test_case1_shape_and_boundaries():
    mesh, flow, _ = load_case1()
    assert (mesh.nods, mesh.neles, mesh.nghosts) == (5916, 5750, 330)
    assert sorted(set(mesh.ntype.tolist())) == [2, 3, 4, 5]
    assert (flow.istart, flow.iaxis, flow.local) == (0, 0, 1)


def test_cold_state_equals_oracle_cold_start():
    mesh, flow, g = load_case1()
    ri = formats.rinit_cold(flow)
    assert ri == float(g["rinit"])
    o = Oracle(mesh, flow, ri)
    o.cold_start()
    assert np.array_equal(o.state(), formats.cold_state(flow, mesh.neles, ri))


def test_oracle_reproduces_case1_fixture():
    mesh, flow, g = load_case1()
    ri = float(g["rinit"])
    o = Oracle(mesh, flow, ri)
    o.set_state(formats.cold_state(flow, mesh.neles, ri))
    hist = o.iterate(int(g["niter"]), int(g["monitor"]))
    assert np.all(_rel(o.state(), g["state"]) <= 1e-14)
    assert np.max(np.abs(hist - g["cdiff"]) / np.abs(g["cdiff"])) <= 1e-14


@pytest.mark.gpu
def test_case1_gpu_matches_oracle():
    """1000 RK4 iterations of the reference's case through the C ABI: Q and the CDIFF
    record of every 100th iteration against the fixture and a live oracle run."""
    from tnsgpu.solver import Solver
    mesh, flow, g = load_case1()
    ri = float(g["rinit"])
    c0 = formats.cold_state(flow, mesh.neles, ri)
    s = Solver(mesh, flow, ri)
    s.upload(c0)
    hist = s.run(int(g["niter"]), int(g["monitor"]))
    q = s.download()
    s.close()
    err, herr = _rel(q, g["state"]), np.max(np.abs(hist - g["cdiff"]) / np.abs(g["cdiff"]))
    print(f"case1 GPU vs oracle: Q rel err {err}, CDIFF history rel err {herr:.3e}")
    assert hist.shape == g["cdiff"].shape
    assert np.all(err <= TOL), err
    assert herr <= TOL
    o = Oracle(mesh, flow, ri)
    o.set_state(c0)
    o.iterate(int(g["niter"]), int(g["monitor"]))
    assert np.all(_rel(q, o.state()) <= TOL)


@pytest.mark.gpu
def test_case1_drop_in_main(tmp_path):
    """The drop-in main on the reference's case files (written back from the fixture in
    the reference's formats, NITER cut to 1000): the monitor line, fort.32, restart.in and
    tec_plot.dat against the oracle."""
    mesh, flow, g = load_case1()
    flow.niter = int(g["niter"])
    formats.write_case(str(tmp_path), mesh, flow)
    r = subprocess.run([os.path.join(os.path.dirname(HERE), "2d-turbulent-navier-stokes_b200",
                                     "mains", "twodturb")], cwd=tmp_path, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if re.match(r"^\s+\d+\s", l)]
    assert [int(l.split()[0]) for l in lines] == [1000]
    assert np.allclose([float(t) for t in lines[0].split()[1:]], g["cdiff"][-1], rtol=1e-5, atol=0)
    assert np.allclose(np.loadtxt(tmp_path / "fort.32"), g["cdiff"][-1], rtol=1e-4)
    cfin, rtred, nps, ri, nold = formats.read_restart(str(tmp_path / "restart.in"), mesh.neles)
    assert np.all(_rel(cfin, g["state"]) <= TOL)
    assert (ri, nold) == (float(g["rinit"]), 1000)
    o = Oracle(mesh, flow, float(g["rinit"]))
    o.set_state(formats.cold_state(flow, mesh.neles, float(g["rinit"])))
    o.iterate(1000, 1000)
    pn, un, vn, tn = o.postprocess()
    tec = open(tmp_path / "tec_plot.dat").read().splitlines()
    vals = np.array([[float(x) for x in l.split()] for l in tec[2:2 + mesh.nods]])
    for col, refv in ((2, un), (3, vn), (4, pn * 1e-5), (7, tn)):
        assert np.max(np.abs(vals[:, col] - refv)) <= TOL * np.max(np.abs(refv)), col


def test_oracle_is_numbering_invariant_on_case1():
    """The oracle on case1 with permuted cell / node ids and rotated local node order
    (tests/meshperm.py) gives the original solution up to summation order: this holds the
    renumbering helper the general-mesh GPU tests use."""
    from meshperm import permute_mesh
    mesh, flow, g = load_case1()
    ri = float(g["rinit"])
    pm, perm = permute_mesh(mesh, seed=1)
    a = Oracle(pm, flow, ri)
    a.set_state(formats.cold_state(flow, pm.neles, ri))
    ha = a.iterate(100, 50)
    b = Oracle(mesh, flow, ri)
    b.set_state(formats.cold_state(flow, mesh.neles, ri))
    hb = b.iterate(100, 50)
    assert np.all(_rel(a.state()[:, perm], b.state()) <= 1e-10)
    assert np.max(np.abs(ha - hb) / np.abs(hb)) <= 1e-10
