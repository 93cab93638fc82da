"""Mixed FP32/FP64 path (precision=1) against the FP64 path on the GPU.

The mixed path stores the stage increments, D, VIS and DT in FP32 and runs the flux,
JST, viscous and source arithmetic in FP32 on top of an FP64 state, FP64 geometry and
FP64 differences, so it follows the FP64 path to FP32 accuracy of the increments.
Tolerances (relative, max-norm per variable, after 50 iterations): 2e-6 for C1 and C4,
1e-4 for the momentum components C2, C3 (small values, the velocity field is where the
FP32 increments show first), 5e-5 for C5 (turbulence variable) on well-conditioned
cases; the CDIFF history to 1e-4.
"""
import numpy as np
import pytest

from tnsgpu import cases, formats
from tnsgpu.solver import Solver

pytestmark = pytest.mark.gpu
TOL = np.array([2e-6, 1e-4, 1e-4, 2e-6, 5e-5])


def rel(a, b):
    return np.max(np.abs(a - b), axis=1) / np.maximum(np.max(np.abs(b), axis=1), 1e-300)


def _pair(mesh, flow, c0, ri, n, mon=10):
    a = Solver(mesh, flow, ri, precision=0)
    a.upload(c0)
    ha = a.run(n, mon)
    b = Solver(mesh, flow, ri, precision=1)
    b.upload(c0)
    hb = b.run(n, mon)
    return a, b, ha, hb


CASES = {
    "ramp": lambda: (cases.ramp_mesh(48, 20), cases.ramp_flow(), "noisy"),
    "nozzle2d": lambda: (cases.nozzle_2d_mesh(40, 18), cases.nozzle_2d_flow(), "cold"),
    "plume_axis_sym": lambda: (cases.nozzle_plume_mesh(64, 24), cases.nozzle_plume_flow(), "cold"),
    "global_dt": lambda: (cases.ramp_mesh(40, 16),
                          formats.Flow(**{**cases.ramp_flow().__dict__, "local": 0}), "noisy"),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_follows_fp64(name):
    mesh, flow, kind = CASES[name]()
    if name == "plume_axis_sym":
        mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    if kind == "noisy":
        c0, ri = cases.noisy_restart_state(flow, mesh.neles)
    else:
        ri = formats.rinit_cold(flow)
        c0 = formats.cold_state(flow, mesh.neles, ri)
    a, b, ha, hb = _pair(mesh, flow, c0, ri, 50)
    err = rel(b.download(), a.download())
    assert np.all(err <= TOL), err
    assert np.max(np.abs(hb - ha) / ha) <= 1e-4
    # frozen terms of the last iteration and the POSTPROCESS primitives
    assert np.all(rel(b.debug(1), a.debug(1)) <= 1e-3)
    assert np.all(rel(b.debug(2), a.debug(2)) <= 1e-6)
    pa, pb = a.primitives(), b.primitives()
    assert np.all(rel(pb[[0, 2, 3]], pa[[0, 2, 3]]) <= 1e-5)


def test_mixed_port_with_injection_profile():
    mesh, flow = cases.port_mesh(40, 16), cases.port_flow()
    mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    ri = formats.rinit_cold(flow)
    c0 = formats.cold_state(flow, mesh.neles, ri)
    a, b, _, _ = _pair(mesh, flow, c0, ri, 30)
    assert np.all(rel(b.download(), a.download()) <= TOL)


def test_mixed_graph_replay_equals_direct_launches_and_parity_alternates():
    mesh, flow = cases.ramp_mesh(40, 20), cases.ramp_flow()
    c0, ri = cases.noisy_restart_state(flow, mesh.neles)
    a = Solver(mesh, flow, ri, precision=1)
    a.upload(c0)
    a.run(7, 0)       # graphs (odd count: ends on the second state buffer)
    a.run(2, 1)       # monitored iterations through their own graphs
    b = Solver(mesh, flow, ri, precision=1)
    b.upload(c0)
    b.profile(True)   # direct launches
    b.run(7, 0)
    b.run(2, 1)
    assert np.array_equal(a.download(), b.download())
    assert np.array_equal(a.primitives(), b.primitives())


@pytest.mark.parametrize("name", sorted(CASES))
def test_mixed_general_mesh_follows_fp64(name):
    """The same cases with their ids shuffled and faces rotated (cases.renumbered_mesh),
    so they take the general-mesh path: its mixed iteration (chunk reference states,
    FP32 slot deviations, FP32 D / VIS / DT) follows its FP64 iteration to the same
    tolerances, the residual record and the POSTPROCESS primitives too."""
    mesh, flow, kind = CASES[name]()
    if name == "plume_axis_sym":
        mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    if kind == "noisy":
        c0, ri = cases.noisy_restart_state(flow, mesh.neles)
    else:
        ri = formats.rinit_cold(flow)
        c0 = formats.cold_state(flow, mesh.neles, ri)
    g, perm = cases.renumbered_mesh(mesh, seed=7)
    q0 = np.empty_like(c0)
    q0[:, perm] = c0
    a, b, ha, hb = _pair(g, flow, q0, ri, 50)
    err = rel(b.download(), a.download())
    print(f"{name} general mesh: mixed vs FP64 {err}")
    assert np.all(err <= TOL), err
    assert np.max(np.abs(hb - ha) / ha) <= 1e-4
    assert np.all(rel(b.primitives(), a.primitives()) <= 1e-4)
    a.close()
    b.close()
