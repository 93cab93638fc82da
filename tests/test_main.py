"""The drop-in main program (twodturb / axiturb): file behaviour of the reference main
(src/solvers/turbnstwod.f90) with the RK4 loop on the GPU, checked against the oracle."""
import os
import re
import subprocess

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tnsgpu import cases, formats

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAINS = os.path.join(ROOT, "2d-turbulent-navier-stokes_b200", "mains")


def _run(exe, cwd):
    return subprocess.run([os.path.join(MAINS, exe)], cwd=cwd, capture_output=True, text=True,
                          timeout=600)


def test_main_rejects_a_mesh_it_cannot_lay_out_before_touching_cuda(tmp_path):
    # one row of cells: the type-3 ghosts have no cell across the opposite face
    xn, yn = np.meshgrid(np.linspace(0.0, 600.0, 7), np.linspace(0.0, 100.0, 2), indexing="ij")
    m = cases.multiblock_mesh([(xn, yn)], lambda x, y: 2 if x == 0.0 else 3)
    f = cases.ramp_flow(10)
    f.istart = 0
    formats.write_case(str(tmp_path), m, f)
    r = _run("twodturb", tmp_path)
    assert r.returncode == 1
    assert "tns_create failed (-3)" in r.stderr


def test_main_reports_missing_flow_in(tmp_path):
    r = _run("twodturb", tmp_path)
    assert r.returncode == 2 and "flow.in" in r.stderr


def test_main_reports_truncated_grid_in(tmp_path):
    m, f = cases.ramp_mesh(6, 4), cases.ramp_flow(10)
    f.istart = 0
    formats.write_case(str(tmp_path), m, f)
    g = tmp_path / "grid.in"
    lines = g.read_text().splitlines()
    g.write_text("\n".join(lines[: len(lines) // 2]) + "\n")  # cut in the middle
    r = _run("twodturb", tmp_path)
    assert r.returncode == 2 and "grid.in" in r.stderr and "end of file" in r.stderr


def test_main_rejects_collapsed_cell_before_touching_cuda(tmp_path):
    m, f = cases.ramp_mesh(6, 4), cases.ramp_flow(10)
    f.istart = 0
    n = m.nod[9] - 1  # cell 10: N2, N3 moved onto N1, N4
    m.x_mm = m.x_mm.copy()
    m.y_mm = m.y_mm.copy()
    m.x_mm[n[1]], m.y_mm[n[1]] = m.x_mm[n[0]], m.y_mm[n[0]]
    m.x_mm[n[2]], m.y_mm[n[2]] = m.x_mm[n[3]], m.y_mm[n[3]]
    m.x, m.y = m.x_mm * 0.001, m.y_mm * 0.001
    formats.write_case(str(tmp_path), m, f)
    r = _run("twodturb", tmp_path)
    assert r.returncode == 1
    assert "tns_create failed (-2)" in r.stderr and "zero volume" in r.stderr


@pytest.mark.gpu
def test_main_reports_nan_in_restart(tmp_path):
    """A NaN in restart.in turns the state non-finite; the main stops with the error
    instead of writing NaN restart files."""
    mesh, flow = cases.ramp_mesh(24, 10), cases.ramp_flow(2000)
    c0, rinit = cases.noisy_restart_state(flow, mesh.neles)
    c0[0, 17] = float("nan")
    formats.write_case(str(tmp_path), mesh, flow)
    formats.write_restart(str(tmp_path / "restart.in"), c0, flow.rtred, flow.npseudo, rinit, 0)
    r = _run("twodturb", tmp_path)
    assert r.returncode == 1
    assert "(-5)" in r.stderr


def _fortran_e(v, d=6):
    """Ew.d of a positive value, as the reference's FORMAT(... E12.6 ...) prints it."""
    if v == 0:
        return "0." + "0" * d + "E+00"
    e = int(np.floor(np.log10(v))) + 1
    mant = round(v / 10.0 ** e * 10 ** d)
    if mant >= 10 ** d:
        e += 1
        mant = round(mant / 10)
    return f"0.{mant:0{d}d}E{'-' if e < 0 else '+'}{abs(e):02d}"


@pytest.mark.gpu
def test_main_files_match_oracle(tmp_path):
    """Restart from a seeded state with NITEROLD=19000 and run 2000 iterations: the
    monitor lines (iterations 20000 and 21000), fort.32, restart     20000.in,
    restart.in and tec_plot.dat follow the oracle."""
    mesh = cases.ramp_mesh(24, 10)
    flow = cases.ramp_flow(2000)
    c0, rinit = cases.noisy_restart_state(flow, mesh.neles)
    formats.write_case(str(tmp_path), mesh, flow)
    formats.write_restart(str(tmp_path / "restart.in"), c0, flow.rtred, flow.npseudo, rinit, 19000)
    r = _run("twodturb", tmp_path)
    assert r.returncode == 0, r.stderr

    o = Oracle(mesh, flow, rinit)
    o.set_state(c0)
    hist1 = o.iterate(1000, 1000)
    s20k = o.state()
    hist2 = o.iterate(1000, 1000)
    ref = o.state()

    lines = [l for l in r.stdout.splitlines() if re.match(r"^\s+\d+\s", l)]
    assert [int(l.split()[0]) for l in lines] == [20000, 21000]
    for line, h in zip(lines, (hist1[0], hist2[0])):
        got = [float(t) for t in line.split()[1:]]
        assert np.allclose(got, h, rtol=1e-5, atol=0)
        assert line.split()[1] == _fortran_e(h[0]) or abs(float(line.split()[1]) / h[0] - 1) < 1e-6
    f32 = np.loadtxt(tmp_path / "fort.32")
    assert np.allclose(f32, np.stack([hist1[0], hist2[0]]), rtol=1e-4)

    c20, *_ = formats.read_restart(str(tmp_path / "restart     20000.in"), mesh.neles)
    cfin, rtred, nps, ri, nold = formats.read_restart(str(tmp_path / "restart.in"), mesh.neles)
    rel = lambda a, b: np.max(np.abs(a - b), axis=1) / np.max(np.abs(b), axis=1)
    assert np.all(rel(c20, s20k) < 1e-10)
    assert np.all(rel(cfin, ref) < 1e-10)
    assert (rtred, nps, ri, nold) == (flow.rtred, flow.npseudo, rinit, 21000)

    pn, un, vn, tn = o.postprocess()
    tec = open(tmp_path / "tec_plot.dat").read().splitlines()
    assert tec[0].strip().startswith("VARIABLES")
    vals = np.array([[float(x) for x in l.split()] for l in tec[2:2 + mesh.nods]])
    assert np.allclose(vals[:, 0], mesh.x, rtol=0, atol=0)
    for col, refv in ((2, un), (3, vn), (4, pn * 1e-5), (7, tn)):
        assert np.max(np.abs(vals[:, col] - refv)) <= 1e-10 * np.max(np.abs(refv)), col
    conn = np.array([[int(x) for x in l.split()] for l in tec[2 + mesh.nods:]])
    assert np.array_equal(conn, mesh.nod)
