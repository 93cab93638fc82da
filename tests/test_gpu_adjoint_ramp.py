"""The compression-ramp gradients (512 x 192 cells, 67 parameters: P0, T0, AMACHINIT and
64 ramp-wall node displacements) of a 500-iteration transient from the cold start,
against central finite differences of the GPU FP64 primal at steps chosen by a step
study.

Step study (central differences, this case):
* P0, AMACHINIT: relative steps 1e-4 .. 1e-2 agree with the adjoint to 1e-14 .. 1e-9.
* T0: the wall force barely depends on T0 (T0/J dJ/dT0 = 8.6e-8), so at a relative step
  of 1e-6 J moves by 1e-13 of itself and the difference is rounding noise (1e-4 .. 1e-3
  off, forward and backward differences apart by 1 %).  At relative steps 1e-3 .. 1e-2
  the difference agrees to about 1e-6, and a Richardson pair (h, 3h) to 2e-7.
* Wall nodes: truncation grows as h^2 above 1e-6 m, rounding below 1e-7 m; at 3e-7 m the
  differences agree to 4e-9 .. 2.5e-6 (the node at i = 260, the ramp's corner, to 3e-5).
The adjoint itself is the exact derivative of the discrete iteration (checked against
autograd of the FP64 restatement in test_gpu_adjoint.py); these tolerances hold the
finite differences, not the adjoint.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N = 500


@pytest.fixture(scope="module")
def ramp():
    from oracle.adjoint_report import CHECK_NODE, _setup
    mesh, flow, sch, space, dy = _setup("cuda")
    return mesh, flow, sch, space, dy, CHECK_NODE


def _central(J, base, h):
    return (J(base + h) - J(base - h)) / (2.0 * h)


def _rel(a, b):
    return abs(a - b) / abs(b)


def test_wall_force_gradient_against_finite_differences(ramp):
    from tnsgpu import adjoint
    mesh, flow, sch, space, dy, node = ramp
    obj = adjoint.wall_force_y
    r = adjoint.transient_gradient(sch, obj, dy=dy.to(sch.device), space=space, niter=N)

    def J_of(which):
        def J(v):
            kw = {"p0": None, "t0": None, "amachinit": None}
            kw[which] = v
            return adjoint.objective_gpu(sch, obj, dy=dy, space=space, niter=N, **kw)
        return J

    def J_node(k):
        def J(v):
            d = dy.clone()
            d[k] = v
            return adjoint.objective_gpu(sch, obj, dy=d, space=space, niter=N)
        return J

    report = {}
    fd = _central(J_of("p0"), flow.p0, 1e-3 * flow.p0)
    report["p0"] = _rel(r["dJ_dp0"], fd)
    assert report["p0"] <= 1e-10
    fd = _central(J_of("amachinit"), flow.amachinit, 1e-3 * flow.amachinit)
    report["amachinit"] = _rel(r["dJ_damachinit"], fd)
    assert report["amachinit"] <= 1e-8

    # T0: J is nearly independent of it, so the step is large
    assert abs(r["dJ_dt0"] * flow.t0 / r["J"]) < 1e-6
    JT = J_of("t0")
    d = {rel: _central(JT, flow.t0, rel * flow.t0) for rel in (3e-2, 1e-2, 3e-3, 1e-3)}
    for rel in (1e-2, 3e-3, 1e-3):
        report[f"t0_h{rel:g}"] = _rel(r["dJ_dt0"], d[rel])
        assert report[f"t0_h{rel:g}"] <= 1e-5, rel
    # Richardson pair (h, 3h) of the O(h^2) central difference
    rich = d[1e-2] + (d[1e-2] - d[3e-2]) / 8.0
    report["t0_richardson"] = _rel(r["dJ_dt0"], rich)
    assert report["t0_richardson"] <= 1e-6

    ddy = r["dJ_ddy"]
    for k, tol in ((node, 1e-5), (10, 1e-5), (40, 1e-5), (63, 1e-7)):
        fd = _central(J_node(k), float(dy[k]), 3e-7)
        report[f"node{k}"] = _rel(float(ddy[k]), fd)
        assert report[f"node{k}"] <= tol, k
    print("wall force, adjoint vs central FD:", {k: f"{v:.2e}" for k, v in report.items()})


def test_total_pressure_loss_gradient_against_finite_differences(ramp):
    from tnsgpu import adjoint
    mesh, flow, sch, space, dy, node = ramp
    obj = adjoint.total_pressure_loss
    r = adjoint.transient_gradient(sch, obj, dy=dy.to(sch.device), space=space, niter=N)

    def J_am(v):
        return adjoint.objective_gpu(sch, obj, amachinit=v, dy=dy, space=space, niter=N)

    def J_t0(v):
        return adjoint.objective_gpu(sch, obj, t0=v, dy=dy, space=space, niter=N)

    def J_corner(v):
        d = dy.clone()
        d[63] = v
        return adjoint.objective_gpu(sch, obj, dy=d, space=space, niter=N)

    e_am = _rel(r["dJ_damachinit"], _central(J_am, flow.amachinit, 3e-3 * flow.amachinit))
    # the loss is nearly independent of T0 too (T0/J dJ/dT0 = 4e-5): the rounding floor of
    # the difference is about 2e-4 at the best step
    e_t0 = _rel(r["dJ_dt0"], _central(J_t0, flow.t0, 3e-2 * flow.t0))
    e_corner = _rel(float(r["dJ_ddy"][63]), _central(J_corner, float(dy[63]), 3e-7))
    print(f"total-pressure loss, adjoint vs central FD: amachinit {e_am:.2e}, t0 {e_t0:.2e}, "
          f"outlet-corner node {e_corner:.2e}")
    assert e_am <= 1e-6
    assert e_t0 <= 1e-3
    assert e_corner <= 1e-5
    # upstream wall nodes do not reach the outlet faces within 500 iterations
    assert np.max(np.abs(r["dJ_ddy"][:40])) <= 1e-12 * np.max(np.abs(r["dJ_ddy"]))
