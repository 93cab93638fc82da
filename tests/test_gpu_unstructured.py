"""General quadrilateral meshes through the C ABI: meshes that are not one structured
i x j block (the reference reads any NOD / NC1..NC4, geometry.f90:31-52) run on the
gather-indexed kernels (csrc/tns_unstructured.cu) and must match the oracle on the same
mesh to <= 1e-10 relative (max-norm per variable), like the structured path.

Meshes: the reference's examples/case1 with its cell and node ids permuted and every
cell's faces starting at another corner (tests/meshperm.py); the same with ids only
permuted (still one block: the structured path with its permutation); a three-block
backward-facing step (cases.backstep_mesh); axisymmetric and port / boundary-layer
variants renumbered the same way."""
import os
import subprocess

import numpy as np
import pytest

from meshperm import permute_mesh
from oracle.pyoracle import Oracle
from test_case1 import load_case1
from tnsgpu import cases, formats
from tnsgpu.solver import Solver

pytestmark = pytest.mark.gpu
TOL = 1e-10
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b):
    a, b = np.atleast_2d(a), np.atleast_2d(b)
    return np.max(np.abs(a - b), axis=1) / np.maximum(np.max(np.abs(b), axis=1), 1e-300)


def _compare(mesh, flow, c0, ri, niter, mon, label):
    s = Solver(mesh, flow, ri)
    s.upload(c0)
    hist = s.run(niter, mon)
    q = s.download()
    prim = s.primitives()
    o = Oracle(mesh, flow, ri)
    o.set_state(c0)
    ref_hist = o.iterate(niter, mon)
    err = rel(q, o.state())
    herr = np.max(np.abs(hist - ref_hist) / np.abs(ref_hist)) if len(ref_hist) else 0.0
    nn = o.nn
    perr = rel(prim[:, :nn], np.stack([o.fetch(k)[:nn] for k in "UVTP"]))
    print(f"{label}: {mesh.neles} cells x {niter} iterations, Q rel err {err}, CDIFF {herr:.3e}, "
          f"primitives {perr.max():.3e}")
    assert hist.shape == ref_hist.shape
    assert np.all(err <= TOL), err
    assert herr <= TOL
    assert np.all(perr <= TOL), perr
    return s, o


def _cold(mesh, flow):
    ri = formats.rinit_cold(flow)
    return formats.cold_state(flow, mesh.neles, ri), ri


def test_case1_renumbered_and_rotated_takes_the_general_path():
    mesh, flow, g = load_case1()
    pm, _ = permute_mesh(mesh, seed=1)
    c0, ri = _cold(pm, flow)
    s, o = _compare(pm, flow, c0, ri, 200, 50, "case1 permuted + rotated")
    # POSTPROCESS node averages and boundary integrals of the last stage
    pn, un, vn, tn = o.postprocess()
    na = s.node_averages()
    for got, ref in zip(na, (pn, un, vn, tn)):
        assert np.max(np.abs(got - ref)) <= TOL * np.max(np.abs(ref))
    s.close()


def test_case1_renumbered_without_rotation_stays_structured():
    mesh, flow, g = load_case1()
    pm, _ = permute_mesh(mesh, seed=2, rotate=False)
    c0, ri = _cold(pm, flow)
    s, _ = _compare(pm, flow, c0, ri, 200, 50, "case1 permuted")
    s.close()


def test_case1_one_iteration_frozen_terms():
    """D, VIS and DT of the first iteration, cell by cell, on the general path."""
    mesh, flow, g = load_case1()
    pm, _ = permute_mesh(mesh, seed=3)
    c0, ri = _cold(pm, flow)
    s = Solver(pm, flow, ri)
    s.upload(c0)
    s.run(1, 0)
    o = Oracle(pm, flow, ri)
    o.set_state(c0)
    o.iterate(1, 0)
    ne = pm.neles
    assert np.all(rel(s.debug(0), np.stack([o.fetch(f"D24{k}")[:ne] for k in range(1, 6)])) < 1e-11)
    assert np.all(rel(s.debug(1), np.stack([o.fetch(k)[:ne] for k in ("VISU", "VISV", "VIST", "VISR")])) < 1e-11)
    assert np.all(rel(s.debug(2), o.fetch("DT")[None, :ne]) < 1e-13)
    s.close()


@pytest.mark.parametrize("local", [1, 0])
def test_backward_facing_step_three_blocks(local):
    mesh, flow = cases.backstep_mesh(32, 96, 24, 12), cases.ramp_flow()
    flow.istart = 0
    flow.local = local
    c0, ri = _cold(mesh, flow)
    s, _ = _compare(mesh, flow, c0, ri, 200, 50, f"backstep LOCAL={local}")
    s.close()


def _bl_ramp():
    m = cases.ramp_mesh(24, 12)
    m.ntype[m.ntype == 2] = 7
    f = cases.ramp_flow()
    f.pinf, f.aminf, f.deltabl = 8.6e5, 0.05, 0.01
    return m, f


@pytest.mark.parametrize("kind", ["port_type4_axis", "plume_type4_axis", "bl_inlet"])
def test_renumbered_axisymmetric_port_and_inlet_cases(kind):
    if kind == "port_type4_axis":
        mesh, flow = cases.port_mesh(40, 16), cases.port_flow()
    elif kind == "plume_type4_axis":
        mesh, flow = cases.nozzle_plume_mesh(48, 20), cases.nozzle_plume_flow()
    else:
        mesh, flow = _bl_ramp()
    if kind != "bl_inlet":
        mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4  # well-conditioned axis
    pm, _ = permute_mesh(mesh, seed=4)
    c0, ri = _cold(pm, flow)
    s, _ = _compare(pm, flow, c0, ri, 20, 10, kind)
    if kind == "port_type4_axis":
        # the port line of each type-6 ghost, walked across a renumbered mesh
        assert np.any(pm.ntype == 6)
    s.close()


def test_drop_in_main_on_a_general_mesh(tmp_path):
    mesh, flow = cases.backstep_mesh(16, 48, 12, 6), cases.ramp_flow(300)
    flow.istart = 0
    formats.write_case(str(tmp_path), mesh, flow)
    r = subprocess.run([os.path.join(os.path.dirname(HERE), "2d-turbulent-navier-stokes_b200", "mains",
                                     "twodturb")], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    cfin, *_ = formats.read_restart(str(tmp_path / "restart.in"), mesh.neles)
    c0, ri = _cold(mesh, flow)
    o = Oracle(mesh, flow, ri)
    o.set_state(c0)
    o.iterate(300, 1000)
    assert np.all(rel(cfin, o.state()) <= TOL)


def _hilbert_chunk_halos(mesh):
    """Halo sizes of the general path's stage chunks (256 cells in Hilbert order of their
    centroids), restated on the host from the layout the library builds."""
    xc, yc = mesh.x[mesh.nod - 1].mean(axis=1), mesh.y[mesh.nod - 1].mean(axis=1)
    N = 1 << 20
    x = ((xc - xc.min()) * ((N - 1) / (xc.max() - xc.min()))).astype(np.int64)
    y = ((yc - yc.min()) * ((N - 1) / (yc.max() - yc.min()))).astype(np.int64)
    d = np.zeros(mesh.neles, dtype=np.uint64)
    s = N // 2
    while s > 0:
        rx, ry = ((x & s) > 0).astype(np.int64), ((y & s) > 0).astype(np.int64)
        d += np.uint64(s) * np.uint64(s) * ((3 * rx) ^ ry).astype(np.uint64)
        flip = (ry == 0) & (rx == 1)
        x[flip], y[flip] = N - 1 - x[flip], N - 1 - y[flip]
        sw = ry == 0
        x[sw], y[sw] = y[sw].copy(), x[sw].copy()
        s //= 2
    order = np.argsort(d, kind="stable")
    new_of = np.empty(mesh.neles, dtype=np.int64)
    new_of[order] = np.arange(mesh.neles)
    nb = mesh.nc[order]  # ids of each renumbered cell's neighbours
    slot = np.where(nb <= mesh.neles, new_of[np.clip(nb, 1, mesh.neles) - 1], mesh.neles + nb)
    halos = []
    for b in range(0, mesh.neles, 256):
        own = np.arange(b, min(b + 256, mesh.neles))
        halos.append(len(np.setdiff1d(np.unique(slot[b:b + 256]), own)))
    return np.array(halos)


def test_full_size_renumbered_nozzle_plume_matches_the_structured_path():
    """The 1024 x 384 nozzle-plume with its ids shuffled and faces rotated runs on the
    general path, whose chunk halos here reach past one thread round (up to 373 slots
    for 256 threads); after 20 iterations it matches the same mesh on the structured
    path (itself held to the oracle at this size) to summation-order rounding, C5 to
    the ill-conditioned axis-wall level."""
    mesh = cases.nozzle_plume_mesh(1024, 384)
    flow = cases.nozzle_plume_flow()
    c0, ri = cases.noisy_restart_state(flow, mesh.neles)
    g, perm = cases.renumbered_mesh(mesh, seed=3)
    halos = _hilbert_chunk_halos(g)
    assert halos.max() > 256, halos.max()
    a = Solver(mesh, flow, ri)
    a.upload(c0)
    ha = a.run(20, 10)
    qa = a.download()
    a.close()
    q0 = np.empty_like(c0)
    q0[:, perm] = c0
    b = Solver(g, flow, ri)
    b.upload(q0)
    hb = b.run(20, 10)
    qb = b.download()[:, perm]
    b.close()
    err = rel(qb, qa)
    herr = np.max(np.abs(hb - ha) / np.abs(ha), axis=0)
    print(f"renumbered nozzle-plume 1024x384: chunk halos mean {halos.mean():.1f} max {halos.max()}, "
          f"Q rel err vs structured {err}, CDIFF {herr}")
    # C5 on this axis-wall case turns roundoff-level input differences into ~1e-4
    # (the oracle's own response to a 1e-15 perturbation, test_gpu_parity.py)
    assert np.all(err[:4] <= TOL) and err[4] <= 1e-4, err
    assert np.all(herr[:4] <= 1e-8) and herr[4] <= 1e-3, herr


def test_general_path_per_kernel_profile():
    """tns_profile on a general mesh: every launch of the iteration timed in order on the
    handle's stream (dissipation, viscous flux with stage 1's field set, the four chunked
    stages), with the same state as an unprofiled run."""
    mesh, flow = cases.backstep_mesh(32, 96, 24, 12), cases.ramp_flow()
    flow.istart = 0
    c0, ri = _cold(mesh, flow)
    a = Solver(mesh, flow, ri)
    a.upload(c0)
    a.run(7, 0)
    b = Solver(mesh, flow, ri)
    b.upload(c0)
    b.profile(True)
    b.run(7, 0)
    assert np.array_equal(a.download(), b.download())
    kt = b.kernel_times()
    assert kt["dissipation"][1] == 7 and kt["viscous"][1] == 7 and kt["stage"][1] == 28
    assert all(kt[k][0] > 0 for k in ("dissipation", "viscous", "stage"))
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_prepare_on_a_general_mesh(precision):
    """tns_prepare on the general path: it launches nothing, and the runs after it equal
    the runs of a handle that captured its graphs at first use, bit for bit (both mixed
    state parities: an odd then an even call)."""
    mesh, flow, g = load_case1()
    pm, _ = permute_mesh(mesh, seed=4)
    c0, ri = _cold(pm, flow)
    out = []
    for prep in (True, False):
        s = Solver(pm, flow, ri, precision=precision)
        s.upload(c0)
        if prep:
            n0 = s.launch_count()
            s.prepare()
            s.prepare()
            assert s.launch_count() == n0
        rec = [s.run(7, 7), s.run(10, 5)]
        out.append((s.download(), rec))
        s.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(a, b)
