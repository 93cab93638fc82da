"""Hand-written discrete adjoint (csrc/tns_adjoint.cuh) against torch.autograd.

The adjoint point functions are compiled for the host (tests/adjoint_host/adj_host.cu)
and run in the order the CUDA kernels run them.  For one RK4 iteration Q_{n+1} = G(Q_n)
of the differentiable restatement (oracle/adjoint_restatement.py) and a random lambda, they must
reproduce lambda dG/dQ_n and the sensitivities to every geometric quantity the iteration
reads (face vectors, volumes, DL, cell / ghost centroids, node coordinates), RTOLERANCE,
S0 and T0 -- the gradients autograd returns for those quantities made leaves."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest
import torch

from oracle.adjoint_restatement import RestatedScheme
from tnsgpu import adjoint, cases, formats
from tnsgpu.solver import make_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _axis_sym(mesh):
    mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    return mesh


CASES = {
    "ramp": lambda: (cases.ramp_mesh(24, 12), cases.ramp_flow()),
    "nozzle2d": lambda: (cases.nozzle_2d_mesh(20, 10), cases.nozzle_2d_flow()),
    "plume_axis": lambda: (_axis_sym(cases.nozzle_plume_mesh(32, 12)), cases.nozzle_plume_flow()),
    "plume_wall_axis": lambda: (cases.nozzle_plume_mesh(28, 10), cases.nozzle_plume_flow()),
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
    mesh, flow = cases.ramp_mesh(nx, ny), cases.ramp_flow()
    mesh.ntype[mesh.ntype == 2] = 7
    return mesh, formats.Flow(**{**flow.__dict__, "pinf": 8.5e5, "aminf": 0.3, "deltabl": 0.1})


@pytest.fixture(scope="session")
def harness(tmp_path_factory):
    if shutil.which("nvcc") is None:
        pytest.skip("nvcc is needed to compile the host harness")
    out = str(tmp_path_factory.mktemp("adjhost") / "libadjhost.so")
    subprocess.run(["nvcc", "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                    os.path.join(ROOT, "tests", "adjoint_host", "adj_host.cu"), "-o", out], check=True)
    L = C.CDLL(out)
    L.adj_host_step.restype = C.c_int
    return L


def _stages(sch, Cold, geo, prm, rtol):
    """RestatedScheme.iteration, keeping the stage states, D, VIS and DT."""
    dt, p = sch.time_step(Cold, geo, prm)
    D = sch.dissipation(Cold, p, dt, geo, rtol)
    Cs, Cc, vis = [Cold], Cold, None
    dtbyvol = dt / geo["vol"]
    for st in range(4):
        full = sch.boundary(sch.primitive(Cc, prm), prm, geo)
        if st == 0:
            vis = sch.viscous(full, geo, prm, rtol)
            vis5 = torch.cat([torch.zeros_like(vis[:1]), vis])
        s3, s5 = sch.source(full, geo, prm)
        R = sch.residual(full, geo, s3, s5)
        dtv = adjoint.ALPHA_RK[st] * dtbyvol
        N = Cold - dtv * (R - vis5 - D)
        n4 = Cold[4] - dtv * adjoint.CFLTURB * (R[4] - vis[3] - D[4])
        n0 = N[0]
        n4 = n0 * adjoint.dmax(torch.zeros_like(n0) + rtol, n4 / n0)
        Cc = torch.cat([N[:4], n4[None]])
        Cs.append(Cc)
    return Cs, D, vis, dt


def _ghost_layout(mesh, sch, geo):
    """Per-ghost arrays in the library's device order: sides 1 (along i), 2 (along j),
    3 (along i), 4 (along j)."""
    ni, nj = sch.ni, sch.nj
    off = {1: 0, 2: ni, 3: ni + nj, 4: 2 * ni + nj}
    ng = 2 * (ni + nj)
    gtype, grank = np.zeros(ng, np.int32), np.zeros(ng, np.int32)
    par = mesh.nparent - 1
    pi, pj = par // nj, par % nj
    for L in range(mesh.nghosts):
        s = int(mesh.nside[L])
        g = off[s] + (pi[L] if s in (1, 3) else pj[L])
        gtype[g] = mesh.ntype[L]
        grank[g] = L
    xg, yg = geo["xc"].detach().numpy(), geo["yc"].detach().numpy()
    gx = np.concatenate([xg[1:-1, 0], xg[-1, 1:-1], xg[1:-1, -1], xg[0, 1:-1]])
    gy = np.concatenate([yg[1:-1, 0], yg[-1, 1:-1], yg[1:-1, -1], yg[0, 1:-1]])
    ginj = np.ones(ng)
    if mesh.inj_scale is not None:
        for L in range(mesh.nghosts):
            s = int(mesh.nside[L])
            ginj[off[s] + (pi[L] if s in (1, 3) else pj[L])] = mesh.inj_scale[L]
    return gtype, grank, np.ascontiguousarray(gx), np.ascontiguousarray(gy), ginj


def _state(mesh, flow, sch, rinit, seed):
    """A developed, non-uniform state: a perturbed cold start after 25 iterations."""
    c0 = formats.cold_state(flow, mesh.neles, rinit)
    rng = np.random.default_rng(seed)
    c0 = c0 * (1 + 2e-2 * rng.uniform(-1, 1, c0.shape))
    c0[2] = 0.05 * c0[1] * rng.uniform(-1, 1, mesh.neles)
    C = torch.tensor(c0.reshape(5, *mesh.shape))
    prm, geo = sch.params(), sch.geometry(sch.x0, sch.y0)
    with torch.no_grad():
        for _ in range(25):
            C = sch.iteration(C, geo, prm)
    return C


def _run(harness, name, seed=0):
    mesh, flow = CASES[name]()
    rinit = formats.rinit_cold(flow)
    sch = RestatedScheme(mesh, flow, rinit=rinit)
    ni, nj = sch.ni, sch.nj
    Cn = _state(mesh, flow, sch, rinit, seed).requires_grad_(True)
    prm = sch.params()
    geo0 = sch.geometry(sch.x0, sch.y0)
    # the geometric quantities, RTOLERANCE, S0 and T0 as leaves
    geo = {k: ([t.detach().clone().requires_grad_(True) for t in v] if isinstance(v, list)
               else v.detach().clone().requires_grad_(True)) for k, v in geo0.items()}
    rtol = torch.tensor(rinit * flow.rtred, dtype=torch.float64, requires_grad=True)
    s0 = prm.s0().detach().clone().requires_grad_(True)
    prm.t0 = prm.t0.detach().clone().requires_grad_(True)
    prm.s0 = lambda: s0
    Cs, D, vis, dt = _stages(sch, Cn, geo, prm, rtol)
    with torch.no_grad():
        ref = sch.iteration(Cn, geo0, sch.params())
    assert torch.equal(Cs[4], ref)
    lam = torch.tensor(np.random.default_rng(seed + 7).normal(size=(5, ni, nj)))
    leaves = [Cn, geo["x"], geo["y"], geo["xc"], geo["yc"], geo["dl"], geo["vol"], *geo["sx"], *geo["sy"],
              rtol, s0, prm.t0]
    grads = torch.autograd.grad(Cs[4], leaves, grad_outputs=lam, allow_unused=True)
    grads = [g if g is not None else torch.zeros_like(l) for g, l in zip(grads, leaves)]
    # the harness
    f = lambda t: np.ascontiguousarray(t.detach().numpy().reshape(-1), np.float64)
    gtype, grank, gx, gy, ginj = _ghost_layout(mesh, sch, geo0)
    x, y = f(sch.x0), f(sch.y0)
    cfldl = f(flow.cfl * geo0["dl"])
    q = [f(c) for c in Cs[:4]]
    Dn, Vn, DTn = f(D), f(vis), f(dt)
    dtmin = float(dt.detach().reshape(-1)[0])
    lam_io = f(lam).copy()
    ncell, npad, nnode = ni * nj, (ni + 2) * (nj + 2), (ni + 1) * (nj + 1)
    sens = np.zeros(8 * ncell + 2 * ncell + 2 * npad + 2 * nnode + ncell + nnode + 2 * ncell)
    prms = make_params(flow, rinit, 0)
    P = lambda a: a.ctypes.data_as(C.c_void_p)
    rc = harness.adj_host_step(C.byref(prms), ni, nj, P(x), P(y), P(cfldl), P(gtype), P(grank), P(gx), P(gy),
                               P(ginj), P(q[0]), P(q[1]), P(q[2]), P(q[3]), P(Dn), P(Vn), P(DTn), C.c_double(dtmin),
                               P(lam_io), 1, P(sens))
    assert rc == 0
    return sch, grads, lam_io, sens


def _split(sens, ni, nj):
    n, npad, nnode = ni * nj, (ni + 2) * (nj + 2), (ni + 1) * (nj + 1)
    out, o = {}, 0
    for k, sz in (("sx", 4 * n), ("sy", 4 * n), ("vol", n), ("dl", n), ("xc", npad), ("yc", npad),
                  ("x", nnode), ("y", nnode), ("rtolc", n), ("rtoln", nnode), ("t0", n), ("s0", n)):
        out[k] = sens[o:o + sz]
        o += sz
    return out


def _close(got, ref, tol=1e-10):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    scale = max(np.max(np.abs(ref)), 1e-300)
    err = np.max(np.abs(got - ref)) / scale if ref.size else 0.0
    return err <= tol, err


@pytest.mark.parametrize("name", sorted(CASES))
def test_state_adjoint_matches_autograd(harness, name):
    sch, grads, lam_n, _ = _run(harness, name)
    ref = grads[0].numpy().reshape(5, -1)
    got = lam_n.reshape(5, -1)
    for m in range(5):
        ok, err = _close(got[m], ref[m])
        assert ok, (name, m, err)


@pytest.mark.parametrize("name", sorted(CASES))
def test_parameter_sensitivities_match_autograd(harness, name):
    sch, grads, _, sens = _run(harness, name)
    ni, nj = sch.ni, sch.nj
    s = _split(sens, ni, nj)
    g = dict(zip(["C", "x", "y", "xc", "yc", "dl", "vol", "sx0", "sx1", "sx2", "sx3", "sy0", "sy1", "sy2", "sy3",
                  "rtol", "s0", "t0"], grads))
    checks = {
        "vol": (s["vol"], g["vol"].numpy().ravel()),
        "dl": (s["dl"], g["dl"].numpy().ravel()),
        "x": (s["x"], g["x"].numpy().ravel()),
        "y": (s["y"], g["y"].numpy().ravel()),
    }
    ring = np.ones((ni + 2, nj + 2), bool)
    ring[0, 0] = ring[0, -1] = ring[-1, 0] = ring[-1, -1] = False
    for k in ("xc", "yc"):
        checks[k] = (s[k].reshape(ni + 2, nj + 2)[ring], g[k].numpy()[ring])
    for k in range(4):
        checks[f"sx{k}"] = (s["sx"][k * ni * nj:(k + 1) * ni * nj], g[f"sx{k}"].numpy().ravel())
        checks[f"sy{k}"] = (s["sy"][k * ni * nj:(k + 1) * ni * nj], g[f"sy{k}"].numpy().ravel())
    checks["rtol"] = ([s["rtolc"].sum() + s["rtoln"].sum()], [float(g["rtol"])])
    checks["s0"] = ([s["s0"].sum()], [float(g["s0"])])
    checks["t0"] = ([s["t0"].sum()], [float(g["t0"])])
    bad = {}
    for k, (got, ref) in checks.items():
        ok, err = _close(got, ref, 1e-9)
        if not ok:
            bad[k] = err
    assert not bad, (name, bad)
