"""Discrete adjoint on the GPU: the differentiable restatement (oracle/adjoint_restatement,
torch FP64 on cuda) against the CUDA FP64 path; the hand-written CUDA adjoint
(tns_adjoint_step, the product's engine) against autograd of the restatement, step by
step and over a transient; and its gradients against central finite differences of the
GPU FP64 path."""
import numpy as np
import pytest
import torch

from oracle.adjoint_restatement import (RestatedScheme, fixed_point_adjoint_torch,
                                        transient_gradient_torch)
from tnsgpu import adjoint, cases, formats
from tnsgpu.solver import Solver

pytestmark = pytest.mark.gpu


def _ramp(nx=64, ny=24, wall=(40, 52)):
    mesh, flow = cases.ramp_mesh(nx, ny), cases.ramp_flow()
    flow.istart = 0
    sch = RestatedScheme(mesh, flow, device="cuda")
    blend = 1.0 - cases.stretch_one_sided(ny, cases.beta_for_first_cell(ny, 0.3, 1e-5))
    space = adjoint.DesignSpace(sch, adjoint.ramp_wall_shape(sch, list(wall), blend))
    return mesh, flow, sch, space


def test_restatement_on_cuda_matches_the_cuda_fp64_path():
    mesh, flow = cases.ramp_mesh(64, 24), cases.ramp_flow()
    c0, rinit = cases.noisy_restart_state(flow, mesh.neles)
    sch = RestatedScheme(mesh, flow, device="cuda", rinit=rinit)
    prm, geo = sch.params(), sch.geometry(sch.x0, sch.y0)
    s = Solver(mesh, flow, rinit, precision=0)
    s.upload(c0)
    s.run(10, 0)
    ref = s.download()
    s.close()
    C = torch.tensor(c0.reshape(5, *mesh.shape), device="cuda")
    with torch.no_grad():
        for _ in range(10):
            C = sch.iteration(C, geo, prm)
    got = C.reshape(5, -1).cpu().numpy()
    rel = np.max(np.abs(got - ref), axis=1) / np.max(np.abs(ref), axis=1)
    assert np.all(rel < 1e-10), rel


def test_gpu_primal_gradient_matches_gpu_finite_differences():
    """Primal and checkpoints from the CUDA FP64 path; FD (relative step 1e-6, node
    displacement 3e-7 m) on the same path.  Tolerance as in tests/test_adjoint.py."""
    mesh, flow, sch, space = _ramp()
    N = 40
    dy0 = torch.zeros(2, dtype=torch.float64)
    r = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy0, space=space, niter=N)
    got = {"p0": r["dJ_dp0"], "t0": r["dJ_dt0"], "am": r["dJ_damachinit"], "dy0": r["dJ_ddy"][0]}
    base = {"p0": flow.p0, "t0": flow.t0, "am": flow.amachinit, "dy0": 1.0}
    eps = np.finfo(np.float64).eps

    def J(p0=None, t0=None, am=None, dy=dy0):
        return adjoint.objective_gpu(sch, adjoint.wall_force_y, p0, t0, am, dy, space, N)

    def fd(which, h):
        if which == "dy0":
            e = torch.tensor([h, 0.0], dtype=torch.float64)
            return (J(dy=dy0 + e) - J(dy=dy0 - e)) / (2 * h)
        b = base[which]
        kw = {"p0": "p0", "t0": "t0", "am": "am"}[which]
        return (J(**{kw: b * (1 + h)}) - J(**{kw: b * (1 - h)})) / (2 * h * b)

    assert abs(J() - r["J"]) <= 1e-12 * abs(r["J"])
    for which in got:
        h = 3e-7 if which == "dy0" else 1e-6
        f1, f2 = fd(which, h), fd(which, 2 * h)
        rounding = 16 * eps * max(abs(r["J"]), 1.0) / (h * base[which])
        tol = max(2e-3 * abs(f1), 2 * abs(f1 - f2), rounding)
        assert abs(got[which] - f1) <= tol, (which, got[which], f1, f2)


def test_autograd_function_backward_is_the_adjoint():
    mesh, flow, sch, space = _ramp(32, 12, wall=(20,))
    theta = torch.tensor([flow.p0, flow.t0, flow.amachinit, 0.0], dtype=torch.float64, requires_grad=True)
    J = adjoint.TransientObjective.apply(theta, sch, adjoint.wall_force_y, space, 10)
    J.backward()
    r = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=torch.zeros(1, dtype=torch.float64),
                                   space=space, niter=10)
    ref = torch.tensor([r["dJ_dp0"], r["dJ_dt0"], r["dJ_damachinit"], r["dJ_ddy"][0]], dtype=torch.float64)
    assert torch.allclose(theta.grad, ref, rtol=1e-12, atol=0.0)
    assert abs(float(J) - r["J"]) <= 1e-12 * abs(r["J"])


def test_graphed_reverse_step_equals_eager():
    mesh, flow, sch, space = _ramp(48, 16, wall=(30,))
    dy = torch.zeros(1, dtype=torch.float64)
    a = transient_gradient_torch(sch, adjoint.wall_force_y, dy=dy, space=space, niter=8, primal="gpu",
                                 graph=True)
    b = transient_gradient_torch(sch, adjoint.wall_force_y, dy=dy, space=space, niter=8, primal="gpu",
                                 states=a["states"], graph=False)
    for k in ("dJ_dp0", "dJ_dt0", "dJ_damachinit"):
        assert abs(a[k] - b[k]) <= 1e-12 * abs(b[k]), (k, a[k], b[k])
    assert abs(a["dJ_ddy"][0] - b["dJ_ddy"][0]) <= 1e-12 * abs(b["dJ_ddy"][0])
    # index_add sums node averages with atomics: compare the adjoint state in max norm
    err = torch.max(torch.abs(a["lambda0"] - b["lambda0"])) / torch.max(torch.abs(b["lambda0"]))
    assert float(err) < 1e-12, float(err)


def _axis_sym(mesh):
    mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    return mesh


STEP_CASES = {
    "ramp": lambda: (cases.ramp_mesh(64, 24), cases.ramp_flow()),
    "plume_axis": lambda: (_axis_sym(cases.nozzle_plume_mesh(64, 24)), cases.nozzle_plume_flow()),
    "plume_wall_axis": lambda: (cases.nozzle_plume_mesh(48, 20), cases.nozzle_plume_flow()),
    "global_dt": lambda: (cases.ramp_mesh(40, 16),
                          formats.Flow(**{**cases.ramp_flow().__dict__, "local": 0})),
    "bl_inlet": lambda: _bl_inlet(48, 20),
    "port": lambda: (cases.port_mesh(48, 16), cases.port_flow()),
    "port_erosive": lambda: (cases.port_mesh(48, 16, seed=4),
                             formats.Flow(**{**cases.port_flow().__dict__, "ancomb": 0.3, "acomb": 1.0e-6})),
}


def _bl_inlet(nx, ny):
    """The ramp with its inlet as a type-7 boundary-layer inflow (M 0.3, 0.1 m layer)."""
    mesh, flow = cases.ramp_mesh(nx, ny), cases.ramp_flow()
    mesh.ntype[mesh.ntype == 2] = 7
    return mesh, formats.Flow(**{**flow.__dict__, "pinf": 8.5e5, "aminf": 0.3, "deltabl": 0.1})


@pytest.mark.parametrize("name", sorted(STEP_CASES))
def test_cuda_adjoint_step_matches_autograd(name):
    """One reverse step of the CUDA adjoint against torch.autograd of the restatement on
    a developed state; the parameter sensitivities through the gradient they give."""
    mesh, flow = STEP_CASES[name]()
    rinit = formats.rinit_cold(flow)
    sch = RestatedScheme(mesh, flow, device="cuda", rinit=rinit)
    space = adjoint.DesignSpace(sch)
    c0 = formats.cold_state(flow, mesh.neles, rinit)
    rng = np.random.default_rng(3)
    c0 = c0 * (1 + 2e-2 * rng.uniform(-1, 1, c0.shape))
    c0[2] = 0.05 * c0[1] * rng.uniform(-1, 1, mesh.neles)
    prm0, geo0 = sch.params(), sch.geometry(sch.x0, sch.y0)
    C = torch.tensor(c0.reshape(5, *mesh.shape), device="cuda")
    with torch.no_grad():
        for _ in range(30):
            C = sch.iteration(C, geo0, prm0)
    lam = torch.tensor(rng.normal(size=(5,) + mesh.shape), device="cuda")
    params, _ = adjoint._leaves(sch, None, None, None, None)
    prm = adjoint.Params(params[0], params[1], params[2], flow)
    Q = C.clone().requires_grad_(True)
    G = sch.iteration(Q, sch.geometry(sch.x0, sch.y0), prm)
    ref = torch.autograd.grad(G, [Q] + params, grad_outputs=lam, allow_unused=True)
    dev = adjoint.DeviceAdjoint(sch, space, prm, None)
    try:
        got = lam.clone().contiguous()
        dev.step(C.contiguous(), got, True)
        sens = dev.sensitivities()
        launches = dev.solver.adjoint_launch_count()
    finally:
        dev.close()
    assert launches > 20
    err = torch.amax(torch.abs(got - ref[0]), dim=(1, 2)) / torch.amax(torch.abs(ref[0]), dim=(1, 2))
    assert float(err.max()) < 1e-10, err
    gp = adjoint._parameter_gradient(sch, space, params, None, sens, None)
    for k in range(3):
        r = float(ref[k + 1]) if ref[k + 1] is not None else 0.0
        assert abs(float(gp[k]) - r) <= 1e-9 * max(abs(r), 1e-300), (k, float(gp[k]), r)


def test_cuda_engine_transient_gradient_matches_torch_engine():
    mesh, flow, sch, space = _ramp(64, 24, wall=(40, 46, 52))
    dy = torch.tensor([1e-5, -2e-5, 5e-6], dtype=torch.float64)
    N = 30
    a = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy, space=space, niter=N)
    b = transient_gradient_torch(sch, adjoint.wall_force_y, dy=dy, space=space, niter=N,
                                 states=a["states"].reshape(N + 1, 5, -1).cpu().numpy())
    assert abs(a["J"] - b["J"]) <= 1e-13 * abs(b["J"])
    # tolerance on each derivative: 1e-9 of itself or of its natural scale |J| / |p|
    # (a derivative that nearly cancels is compared at the scale of its terms)
    for k, p in (("dJ_dp0", flow.p0), ("dJ_dt0", flow.t0), ("dJ_damachinit", flow.amachinit)):
        tol = 1e-9 * max(abs(b[k]), abs(b["J"]) / p)
        assert abs(a[k] - b[k]) <= tol, (k, a[k], b[k])
    assert np.allclose(a["dJ_ddy"], b["dJ_ddy"], rtol=1e-9, atol=1e-9 * np.max(np.abs(b["dJ_ddy"])))
    err = torch.max(torch.abs(a["lambda0"] - b["lambda0"])) / torch.max(torch.abs(b["lambda0"]))
    assert float(err) < 1e-10, float(err)


def test_cuda_fixed_point_adjoint_matches_torch_engine():
    mesh, flow, sch, space = _ramp(48, 16, wall=(30,))
    s = Solver(mesh, flow, float(sch.rtol(sch.params()) / flow.rtred), precision=0)
    s.upload(sch.cold_state(sch.params()).reshape(5, -1).cpu().numpy())
    s.run(200, 0)
    qstar = torch.tensor(s.download().reshape(5, *mesh.shape), device="cuda")
    s.close()
    dy = torch.zeros(1, dtype=torch.float64)
    a = adjoint.fixed_point_adjoint(sch, adjoint.wall_force_y, qstar, niter=20, dy=dy, space=space)
    b = fixed_point_adjoint_torch(sch, adjoint.wall_force_y, qstar, niter=20, dy=dy, space=space)
    assert np.allclose(a["residual_history"], b["residual_history"], rtol=1e-8)
    for k, p in (("dJ_dp0", flow.p0), ("dJ_dt0", flow.t0), ("dJ_damachinit", flow.amachinit)):
        tol = 1e-9 * max(abs(b[k]), abs(b["J"]) / p)
        assert abs(a[k] - b[k]) <= tol, (k, a[k], b[k])
    assert abs(a["dJ_ddy"][0] - b["dJ_ddy"][0]) <= 1e-9 * abs(b["dJ_ddy"][0])


def test_cuda_adjoint_step_is_deterministic():
    """Repeated sweeps, and a sweep whose next checkpoint's forward values are computed
    beside each reverse (tns_adjoint_step_next), give bitwise the same results."""
    mesh, flow, sch, space = _ramp(64, 24)
    prm = sch.params()
    dev = adjoint.DeviceAdjoint(sch, space, prm, None)
    try:
        st = dev.primal(sch.cold_state(prm).contiguous(), 12)
        lam0 = torch.tensor(np.random.default_rng(5).normal(size=(5,) + mesh.shape), device="cuda")
        outs = []
        for pipelined in (False, False, True):
            lam = lam0.clone()
            for n in range(11, -1, -1):
                dev.step(st[n], lam, True, q_next=st[n - 1] if pipelined and n > 0 else None)
            s = dev.sensitivities()
            outs.append((lam, s["vol"], s["sx"][2]))
    finally:
        dev.close()
    for o in outs[1:]:
        assert all(torch.equal(a, b) for a, b in zip(outs[0], o))


def test_frozen_adjoint_steps_equal_full_steps():
    """TNS_ADJ_FROZEN reuses the forward values of the previous call's state: bitwise the
    same lambda and sensitivities as full steps at that state."""
    mesh, flow, sch, space = _ramp(64, 24)
    prm = sch.params()
    dev = adjoint.DeviceAdjoint(sch, space, prm, None)
    try:
        q = dev.primal(sch.cold_state(prm).contiguous(), 40)[40].contiguous()
        lam0 = torch.tensor(np.random.default_rng(9).normal(size=(5,) + mesh.shape), device="cuda")
        runs = []
        for frozen in (False, True):
            lam = lam0.clone()
            dev.step(q, lam, False)
            for _ in range(3):
                dev.step(q, lam, False, frozen=frozen)
            dev.step(q, lam, True, frozen=frozen)
            runs.append((lam, dev.sensitivities()["sx"][1]))
    finally:
        dev.close()
    assert torch.equal(runs[0][0], runs[1][0]) and torch.equal(runs[0][1], runs[1][1])


def test_bounded_memory_sweep_equals_stored_states():
    """max_states: snapshots at bisection points, segments recomputed from them (the
    primal is deterministic, so the gradient is the same bit for bit)."""
    mesh, flow, sch, space = _ramp(48, 16, wall=(30,))
    dy = torch.tensor([2e-5], dtype=torch.float64)
    N = 30
    a = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy, space=space, niter=N)
    b = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy, space=space, niter=N,
                                   max_states=4)
    assert b["states"] is None and b["recomputed_iterations"] > N
    assert a["J"] == b["J"]
    for k in ("dJ_dp0", "dJ_dt0", "dJ_damachinit"):
        assert a[k] == b[k], (k, a[k], b[k])
    assert np.array_equal(a["dJ_ddy"], b["dJ_ddy"])
    assert torch.equal(a["lambda0"], b["lambda0"])


def test_scalar_sensitivities_equal_full_ones():
    """Without node displacements the sweep accumulates only the RTOLERANCE, T0 and S0
    sensitivities (TNS_ADJ_SCALARS): the P0, T0, AMACHINIT gradient is unchanged."""
    mesh, flow, sch, space = _ramp(48, 16, wall=(30,))
    N = 20
    a = adjoint.transient_gradient(sch, adjoint.total_pressure_loss, dy=torch.zeros(1, dtype=torch.float64),
                                   space=space, niter=N)
    b = adjoint.transient_gradient(sch, adjoint.total_pressure_loss, niter=N)
    for k in ("J", "dJ_dp0", "dJ_dt0", "dJ_damachinit"):
        assert a[k] == b[k], (k, a[k], b[k])


def test_adjoint_abi_errors_leave_the_handle_usable():
    """Refusals are return codes with a message: a mixed-precision handle, a frozen step
    before any full step, a sensitivity buffer of the wrong size."""
    import ctypes as C
    from tnsgpu import _lib
    mesh, flow = cases.ramp_mesh(32, 12), cases.ramp_flow()
    rinit = formats.rinit_cold(flow)
    mx = Solver(mesh, flow, rinit, precision=1)
    try:
        assert mx.L.tns_adjoint_enable(mx.h) == _lib.TNS_ERR_ARG
        assert b"FP64" in mx.L.tns_last_error(mx.h)
    finally:
        mx.close()
    s = Solver(mesh, flow, rinit, precision=0)
    try:
        q = torch.tensor(formats.cold_state(flow, mesh.neles, rinit), device="cuda").contiguous()
        lam = torch.ones_like(q)
        torch.cuda.synchronize()
        rc = s.L.tns_adjoint_step(s.h, C.c_void_p(q.data_ptr()), C.c_void_p(lam.data_ptr()), 2)
        assert rc == _lib.TNS_ERR_STATE, rc
        n = int(s.L.tns_adjoint_sensitivity_size(s.h))
        buf = np.zeros(n + 1)
        assert s.L.tns_adjoint_sensitivities(s.h, buf.ctypes.data, n + 1, 0) == _lib.TNS_ERR_ARG
        s.adjoint_step(q.data_ptr(), lam.data_ptr(), True)
        s.synchronize()
        assert torch.isfinite(lam).all()
        assert np.isfinite(s.adjoint_sensitivities()).all()
    finally:
        s.close()


def test_recorded_forward_values_equal_recomputed():
    """tns_adjoint_record's primal equals tns_enqueue's bit for bit, and reverse steps
    reading the records equal recomputing ones."""
    mesh, flow, sch, space = _ramp(48, 16, wall=(30,))
    dy = torch.tensor([1e-5], dtype=torch.float64)
    N = 25
    a = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy, space=space, niter=N, record=True)
    b = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy, space=space, niter=N, record=False)
    assert torch.equal(a["states"], b["states"])
    for k in ("J", "dJ_dp0", "dJ_dt0", "dJ_damachinit"):
        assert a[k] == b[k], (k, a[k], b[k])
    assert np.array_equal(a["dJ_ddy"], b["dJ_ddy"])
    assert torch.equal(a["lambda0"], b["lambda0"])
