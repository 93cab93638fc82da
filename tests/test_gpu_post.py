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
