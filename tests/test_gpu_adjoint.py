"""Discrete adjoint on the GPU: the differentiable restatement (torch FP64 on cuda)
against the CUDA FP64 path, and gradients whose primal runs through the C ABI against
central finite differences of that same GPU path."""
import numpy as np
import pytest
import torch

from tnsgpu import adjoint, cases, formats
from tnsgpu.solver import Solver

pytestmark = pytest.mark.gpu


def _ramp(nx=64, ny=24, wall=(40, 52)):
    mesh, flow = cases.ramp_mesh(nx, ny), cases.ramp_flow()
    flow.istart = 0
    sch = adjoint.Scheme(mesh, flow, device="cuda")
    blend = 1.0 - cases.stretch_one_sided(ny, cases.beta_for_first_cell(ny, 0.3, 1e-5))
    space = adjoint.DesignSpace(sch, adjoint.ramp_wall_shape(sch, list(wall), blend))
    return mesh, flow, sch, space


def test_restatement_on_cuda_matches_the_cuda_fp64_path():
    mesh, flow = cases.ramp_mesh(64, 24), cases.ramp_flow()
    c0, rinit = cases.noisy_restart_state(flow, mesh.neles)
    sch = adjoint.Scheme(mesh, flow, device="cuda", rinit=rinit)
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
    r = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy0, space=space, niter=N, primal="gpu")
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
                                   space=space, niter=10, primal="gpu")
    ref = torch.tensor([r["dJ_dp0"], r["dJ_dt0"], r["dJ_damachinit"], r["dJ_ddy"][0]], dtype=torch.float64)
    assert torch.allclose(theta.grad, ref, rtol=1e-12, atol=0.0)
    assert abs(float(J) - r["J"]) <= 1e-12 * abs(r["J"])


def test_graphed_reverse_step_equals_eager():
    mesh, flow, sch, space = _ramp(48, 16, wall=(30,))
    dy = torch.zeros(1, dtype=torch.float64)
    a = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy, space=space, niter=8, primal="gpu",
                                   graph=True)
    b = adjoint.transient_gradient(sch, adjoint.wall_force_y, dy=dy, space=space, niter=8, primal="gpu",
                                   states=a["states"], graph=False)
    for k in ("dJ_dp0", "dJ_dt0", "dJ_damachinit"):
        assert abs(a[k] - b[k]) <= 1e-12 * abs(b[k]), (k, a[k], b[k])
    assert abs(a["dJ_ddy"][0] - b["dJ_ddy"][0]) <= 1e-12 * abs(b["dJ_ddy"][0])
    # index_add sums node averages with atomics: compare the adjoint state in max norm
    err = torch.max(torch.abs(a["lambda0"] - b["lambda0"])) / torch.max(torch.abs(b["lambda0"]))
    assert float(err) < 1e-12, float(err)
