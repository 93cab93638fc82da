"""POSTPROCESS node averages and boundary integrals computed on the GPU, against the
oracle's POSTPROCESS (solver_state.f90:237-281) and the host-side objectives."""
import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tnsgpu import cases, formats, objectives
from tnsgpu.solver import Solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_node_averages_and_integrals(precision):
    mesh, flow = cases.nozzle_2d_mesh(30, 14), cases.nozzle_2d_flow()
    ri = formats.rinit_cold(flow)
    c0 = formats.cold_state(flow, mesh.neles, ri)
    s = Solver(mesh, flow, ri, precision=precision)
    s.upload(c0)
    s.run(40, 0)
    o = Oracle(mesh, flow, ri)
    o.set_state(c0)
    o.iterate(40, 0)
    ref = np.stack(o.postprocess())
    got = s.node_averages()
    tol = 1e-10 if precision == 0 else 1e-6
    for k in (0, 2, 3):  # P, V, T relative to their scale; U checked below
        assert np.max(np.abs(got[k] - ref[k])) <= tol * np.max(np.abs(ref[k])), k
    assert np.max(np.abs(got[1] - ref[1])) <= 1e-4 * np.max(np.abs(ref[1])) if precision else \
        np.max(np.abs(got[1] - ref[1])) <= 1e-10 * np.max(np.abs(ref[1]))
    prims = s.primitives()
    for btype, side in ((5, 3), (3, 2), (0, 4), (0, 0)):
        gi = s.boundary_integrals(btype, side)
        sel_side = None if side == 0 else side
        wt = None if btype == 0 else btype
        fx, fy = objectives.wall_force(mesh, prims, flow.amol, flow.iaxis, side=sel_side,
                                       wall_type=wt) if wt else _force_any(mesh, prims, flow, sel_side)
        assert abs(gi[0] - fx) <= 1e-12 * max(abs(fx), 1e-300) + 1e-12
        assert abs(gi[1] - fy) <= 1e-12 * max(abs(fy), 1.0)
    mdot = objectives.outlet_mass_flow(mesh, prims, flow.amol, flow.iaxis, side=2)
    assert abs(s.boundary_integrals(0, 2)[2] - mdot) <= 1e-12 * abs(mdot)


def _force_any(mesh, prims, flow, side):
    _, _, pf, _, _ = objectives._face_state(mesh, prims, flow.amol)
    sx, sy, _, _ = objectives.face_vectors(mesh, flow.iaxis)
    sel = np.ones(mesh.nghosts, bool) if side is None else mesh.nside == side
    return np.sum(pf[sel] * sx[sel]), np.sum(pf[sel] * sy[sel])


def _host_tp_sums(mesh, prims, flow, sel):
    """Host restatement of tns_total_pressure_sums over the bc.in lines ``sel``."""
    uf, vf, pf, rhof, tf = objectives._face_state(mesh, prims, flow.amol)
    sx, sy, _, _ = objectives.face_vectors(mesh, flow.iaxis)
    rr = objectives.RUNIV / flow.amol
    g = flow.gama
    m2 = (uf * uf + vf * vf) / (g * rr * tf)
    p0 = pf * (1.0 + 0.5 * (g - 1.0) * m2) ** (g / (g - 1.0))
    md = np.abs(rhof * (uf * sx + vf * sy))
    return np.array([np.sum((p0 * md)[sel]), np.sum(md[sel])])


@pytest.mark.parametrize("kind", ["nozzle2d", "plume_axi", "backstep_general"])
def test_face_states_and_total_pressure_loss_on_the_gpu(kind):
    """tns_boundary_face_states (the wall pressure distribution) and
    tns_total_pressure_sums (the total-pressure loss objective) against the host
    objectives on the same downloaded primitives, on a structured 2-D channel, an
    axisymmetric mesh and a general (three-block) mesh."""
    if kind == "nozzle2d":
        mesh, flow = cases.nozzle_2d_mesh(30, 14), cases.nozzle_2d_flow()
    elif kind == "plume_axi":
        mesh, flow = cases.nozzle_plume_mesh(48, 20), cases.nozzle_plume_flow()
        mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    else:
        mesh, flow = cases.backstep_mesh(16, 48, 12, 6), cases.ramp_flow()
        flow.istart = 0
    ri = formats.rinit_cold(flow)
    s = Solver(mesh, flow, ri)
    s.upload(formats.cold_state(flow, mesh.neles, ri))
    s.run(60, 0)
    prims = s.primitives()
    fs = s.boundary_face_states()
    ref = np.stack(objectives._face_state(mesh, prims, flow.amol))  # U, V, P, RHO, T
    for k in range(5):
        assert np.max(np.abs(fs[k] - ref[k])) <= 1e-13 * np.max(np.abs(ref[k])) + 1e-300, k
    walls = mesh.ntype == 5
    assert np.array_equal(s.wall_pressure(5), fs[2][walls])
    # inlet = the type-2 faces, outlet = the type-3 faces (valid on any numbering)
    for btype in (2, 3):
        got = s.total_pressure_sums(btype, 0)
        want = _host_tp_sums(mesh, prims, flow, mesh.ntype == btype)
        assert np.all(np.abs(got - want) <= 1e-12 * np.abs(want)), (btype, got, want)
    loss = s.total_pressure_loss((2, 0), (3, 0))
    i, o = _host_tp_sums(mesh, prims, flow, mesh.ntype == 2), _host_tp_sums(mesh, prims, flow, mesh.ntype == 3)
    want = 1.0 - (o[0] / o[1]) / (i[0] / i[1])
    assert abs(loss - want) <= 1e-10 * max(abs(want), 1e-12), (loss, want)
    s.close()
