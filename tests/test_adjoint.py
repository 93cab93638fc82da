"""Discrete adjoint: the differentiable restatement of one RK4 iteration
(oracle/adjoint_restatement.py, the CUDA adjoint's checker) against the oracle, the checkpointed reverse sweep against plain autograd, the gradients
against central finite differences of the oracle, and the fixed-point adjoint against
the truncated Neumann series it sums.  CPU only (torch FP64 on the host)."""
import dataclasses

import numpy as np
import pytest
import torch

from oracle.adjoint_restatement import (RestatedScheme, fixed_point_adjoint_torch,
                                        transient_gradient_torch)
from oracle.pyoracle import Oracle
from tnsgpu import adjoint, cases, formats


def _axis_sym(mesh):
    mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    return mesh


CASES = {
    "ramp": lambda: (cases.ramp_mesh(24, 12), cases.ramp_flow()),
    "nozzle2d": lambda: (cases.nozzle_2d_mesh(20, 10), cases.nozzle_2d_flow()),
    "plume_axis": lambda: (_axis_sym(cases.nozzle_plume_mesh(32, 12)), cases.nozzle_plume_flow()),
    "global_dt": lambda: (cases.ramp_mesh(20, 10),
                          formats.Flow(**{**cases.ramp_flow().__dict__, "local": 0})),
    "bl_inlet": lambda: _bl_inlet(24, 12),
    "port": lambda: (cases.port_mesh(16, 8), cases.port_flow()),
    "port_burn_law": lambda: (cases.port_mesh(16, 8, seed=3),
                              formats.Flow(**{**cases.port_flow().__dict__, "ancomb": 0.3})),
    # a burn rate small enough for the erosive branch (GVAL > GTH) at every port ghost
    "port_erosive": lambda: (cases.port_mesh(16, 8, seed=4),
                             formats.Flow(**{**cases.port_flow().__dict__, "ancomb": 0.3, "acomb": 1.0e-6})),
}


def _bl_inlet(nx, ny):
    """The ramp with its inlet as a type-7 boundary-layer inflow (M 0.3, 0.1 m layer)."""
    mesh, flow = cases.ramp_mesh(nx, ny), cases.ramp_flow()
    mesh.ntype[mesh.ntype == 2] = 7
    return mesh, formats.Flow(**{**flow.__dict__, "pinf": 8.5e5, "aminf": 0.3, "deltabl": 0.1})


@pytest.mark.parametrize("name", sorted(CASES))
def test_restatement_matches_oracle(name):
    mesh, flow = CASES[name]()
    rinit = formats.rinit_cold(flow)
    c0 = formats.cold_state(flow, mesh.neles, rinit)
    c0[0] *= 1 + 1e-3 * np.random.default_rng(1).uniform(-1, 1, mesh.neles)
    sch = RestatedScheme(mesh, flow, rinit=rinit)
    prm, geo = sch.params(), sch.geometry(sch.x0, sch.y0)
    o = Oracle(mesh, flow, rinit)
    o.set_state(c0)
    o.iterate(20, 0)
    C = torch.tensor(c0.reshape(5, *mesh.shape))
    with torch.no_grad():
        for _ in range(20):
            C = sch.iteration(C, geo, prm)
    ref = o.state()
    rel = np.max(np.abs(C.reshape(5, -1).numpy() - ref), axis=1) / np.max(np.abs(ref), axis=1)
    assert np.all(rel < 1e-12), rel


def test_unsupported_boundary_types_are_refused():
    mesh, flow = cases.ramp_mesh(16, 8), cases.ramp_flow()
    mesh.ntype[0] = 9
    with pytest.raises(NotImplementedError):
        adjoint.Scheme(mesh, flow)


def _ramp_space(nx=24, ny=12, wall=(14, 18)):
    mesh, flow = cases.ramp_mesh(nx, ny), cases.ramp_flow()
    flow.istart = 0
    sch = RestatedScheme(mesh, flow)
    blend = 1.0 - cases.stretch_one_sided(ny, cases.beta_for_first_cell(ny, 0.3, 1e-5))
    space = adjoint.DesignSpace(sch, adjoint.ramp_wall_shape(sch, list(wall), blend))
    return mesh, flow, sch, space


def test_checkpointed_sweep_equals_autograd_through_all_iterations():
    mesh, flow, sch, space = _ramp_space(12, 8, wall=(8,))
    N = 6
    r = transient_gradient_torch(sch, adjoint.wall_force_y, dy=torch.zeros(1, dtype=torch.float64),
                                 space=space, niter=N, primal="torch")
    th = [torch.tensor(v, dtype=torch.float64, requires_grad=True) for v in (flow.p0, flow.t0, flow.amachinit)]
    dy = torch.zeros(1, dtype=torch.float64, requires_grad=True)
    prm = adjoint.Params(th[0], th[1], th[2], flow)
    x, y = space.coords(dy)
    geo = sch.geometry(x, y)
    C = sch.cold_state(prm)
    for _ in range(N):
        C = sch.iteration(C, geo, prm)
    g = torch.autograd.grad(adjoint.wall_force_y(sch, C, geo, prm), th + [dy])
    got = [r["dJ_dp0"], r["dJ_dt0"], r["dJ_damachinit"], r["dJ_ddy"][0]]
    for a, b in zip(got, g):
        assert abs(a - float(b)) <= 1e-9 * abs(float(b)), (a, float(b))


def _fd_oracle(mesh, flow, sch, space, objective, N, which, h, dy0):
    def J(p0=flow.p0, t0=flow.t0, am=flow.amachinit, dy=dy0):
        prm = sch.params(p0, t0, am)
        c0 = sch.cold_state(prm).reshape(5, -1).numpy()
        x, y = space.coords(dy)
        m = dataclasses.replace(mesh, x=x.numpy().ravel().copy(), y=y.numpy().ravel().copy())
        f = dataclasses.replace(flow, p0=p0, t0=t0, amachinit=am)
        o = Oracle(m, f, float(sch.rtol(prm) / flow.rtred))
        o.set_state(c0)
        o.iterate(N, 0)
        C = torch.tensor(o.state().reshape(5, *mesh.shape))
        return float(objective(sch, C, sch.geometry(x, y), prm))

    if which in ("p0", "t0", "am"):
        base = {"p0": flow.p0, "t0": flow.t0, "am": flow.amachinit}[which]
        return (J(**{which: base + h * base}) - J(**{which: base - h * base})) / (2 * h * base)
    k = int(which[2:])
    e = torch.zeros_like(dy0)
    e[k] = h
    return (J(dy=dy0 + e) - J(dy=dy0 - e)) / (2 * h)


@pytest.mark.parametrize("objective", ["wall_force_y", "total_pressure_loss"])
def test_gradient_matches_central_differences_of_the_oracle(objective):
    """Relative FD step 1e-6 (node displacements: 3e-7 m).  The scheme has switches
    (the PHI > 0 source branch, |.| in the JST sensors and BCs), so FD is noisy at this
    step: agreement is required to 2e-3 relative, or to the FD's own change between
    steps h and 2h, or to the FD's rounding bound 16 eps max(|J|, 1) / h (the loss is
    formed as 1 - ratio, so its absolute rounding is eps), whichever is largest."""
    mesh, flow, sch, space = _ramp_space()
    N = 20
    obj = getattr(adjoint, objective)
    dy0 = torch.zeros(2, dtype=torch.float64)
    r = transient_gradient_torch(sch, obj, dy=dy0, space=space, niter=N, primal="torch")
    got = {"p0": r["dJ_dp0"], "t0": r["dJ_dt0"], "am": r["dJ_damachinit"],
           "dy0": r["dJ_ddy"][0], "dy1": r["dJ_ddy"][1]}
    base = {"p0": flow.p0, "t0": flow.t0, "am": flow.amachinit, "dy0": 1.0, "dy1": 1.0}
    eps = np.finfo(np.float64).eps
    for which in got:
        h = 3e-7 if which.startswith("dy") else 1e-6
        fd1 = _fd_oracle(mesh, flow, sch, space, obj, N, which, h, dy0)
        fd2 = _fd_oracle(mesh, flow, sch, space, obj, N, which, 2 * h, dy0)
        rounding = 16 * eps * max(abs(r["J"]), 1.0) / (h * base[which])
        tol = max(2e-3 * abs(fd1), 2 * abs(fd1 - fd2), rounding)
        assert abs(got[which] - fd1) <= tol, (objective, which, got[which], fd1, fd2)


def test_fixed_point_adjoint_sums_the_neumann_series():
    """K sweeps of lambda <- dJ/dQ + lambda A (A = dG/dQ at a frozen state) give
    dJ/dQ (I + A + ... + A^K); checked against the dense Jacobian on a tiny mesh."""
    mesh, flow, sch, space = _ramp_space(6, 4, wall=(4,))
    prm, geo = sch.params(), sch.geometry(sch.x0, sch.y0)
    Q = sch.cold_state(prm)
    with torch.no_grad():
        for _ in range(3):
            Q = sch.iteration(Q, geo, prm)
    K = 4
    r = fixed_point_adjoint_torch(sch, adjoint.wall_force_y, Q, niter=K)
    n = Q.numel()
    A = torch.autograd.functional.jacobian(lambda q: sch.iteration(q.reshape(Q.shape), geo, prm).reshape(-1),
                                           Q.reshape(-1))
    Qg = Q.clone().requires_grad_(True)
    (dj,) = torch.autograd.grad(adjoint.wall_force_y(sch, Qg, geo, prm), [Qg])
    lam = dj.reshape(1, n)
    acc = lam.clone()
    for _ in range(K):
        lam = lam @ A
        acc = acc + lam
    ref = acc.reshape(Q.shape)
    err = torch.max(torch.abs(r["lambda"] - ref)) / torch.max(torch.abs(ref))
    assert float(err) < 1e-10, float(err)
    assert len(r["residual_history"]) == K
