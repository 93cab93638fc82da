"""FP64 PyTorch restatement of one RK4 iteration -- TEST INFRASTRUCTURE: the checker of
the hand-written CUDA discrete adjoint (csrc/tns_adjoint.*) and of the oracle.  Only
tests/, __graft_entry__.smoke() and the adjoint reports in this directory import it;
the product's adjoint (tnsgpu/adjoint.py) is the CUDA engine alone.

``RestatedScheme`` extends the product's ``tnsgpu.adjoint.Scheme`` (geometry, primitive
variables, APPLY_BOUNDARY, objectives) with the rest of one iteration of
turbnstwod.f90:95-146 -- DT (turbnstwod.f90:97-114), DISSIPATION
(solver_state.f90:70-225), COMPUTE_VISCOUS with the order-dependent node averages
(viscous.f90:29-217), COMPUTE_SOURCE_TERMS (source_terms.f90:24-104), COMPUTE_RESIDUAL
and UPDATE_SOLUTION (residual.f90:23-83) -- as vectorised FP64 tensor code, so that
torch.autograd differentiates the iteration exactly.  It matches the C oracle to 1e-18
after 20 iterations (tests/test_adjoint.py).  ``transient_gradient_torch`` and
``fixed_point_adjoint_torch`` are the autograd reverse sweeps the CUDA engine is
checked against.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, List, Optional

import numpy as np
import torch

from tnsgpu.adjoint import (ALPHA_RK, BETA_T, ALPHA_T, AMU_THRESH, C02, C04, CFLTURB, CMU,
                            CONST1, CONST2, CONST3, C_, F_, G_, NW_, P_, SUTH, T_, U_, V_,
                            YAXIS_THRESH, DesignSpace, Params, Scheme, _mesh_with_coords,
                            _pad, _safe_sqrt, dmax, dmin, primal_gpu)
from tnsgpu.formats import Mesh


class RestatedScheme(Scheme):
    """The product Scheme plus the whole RK4 iteration (``iteration``)."""

    def __init__(self, mesh: Mesh, flow, device="cpu", rinit: Optional[float] = None):
        super().__init__(mesh, flow, device=device, rinit=rinit)
        self._node_average_matrices(mesh)

    @staticmethod
    def _nb(a):
        """The four neighbours NC1..NC4 (j-1, i+1, j+1, i-1) of every cell of a padded field
        (or stack of fields)."""
        return a[..., 1:-1, :-2], a[..., 2:, 1:-1], a[..., 1:-1, 2:], a[..., :-2, 1:-1]

    def _node_average_matrices(self, mesh: Mesh):
        """NODAL_AVERAGE (viscous.f90:40-124) as sparse maps from the cell values and
        the ghost values (ghosts in bc.in order) to the nodes.  The Fortran visits the
        elements in id order, then the ghosts in bc.in order; a type-4 ghost zeroes VN,
        a type-5 ghost zeroes UN, VN and sets RN = RTOLERANCE*RTRED, after which later
        contributions add to the reset value; every visit counts.  Per node and
        component the average is therefore (base + sum of the contributions after the
        last reset) / count, which these matrices encode."""
        ni, nj = self.ni, self.nj
        nn = (ni + 1) * (nj + 1)
        neles, ng = mesh.neles, mesh.nghosts
        # contribution lists per node: (kind, index) with kind 0 = cell, 1 = ghost line
        contrib = [[] for _ in range(nn)]
        for c in range(neles):
            for k in range(4):
                contrib[mesh.nod[c, k] - 1].append((0, c))
        resets = {"u": [-1] * nn, "v": [-1] * nn, "r": [-1] * nn}
        for g in range(ng):
            p = mesh.nparent[g] - 1
            s = mesh.nside[g]
            n1 = mesh.nod[p, s - 1] - 1
            n2 = mesh.nod[p, s % 4] - 1
            for n in (n1, n2):
                contrib[n].append((1, g))
                pos = len(contrib[n]) - 1
                if mesh.ntype[g] == 4:
                    resets["v"][n] = pos
                elif mesh.ntype[g] == 5:
                    resets["u"][n] = resets["v"][n] = resets["r"][n] = pos
        # ghost line -> flat index into the padded (ni+2, nj+2) ghost ring
        par = mesh.nparent - 1
        pi, pj = par // nj, par % nj
        side = mesh.nside
        gi = np.where(side == 2, pi + 2, np.where(side == 4, pi, pi + 1))
        gj = np.where(side == 1, pj, np.where(side == 3, pj + 2, pj + 1))
        gflat = gi * (nj + 2) + gj
        cflat = lambda c: ((c // nj) + 1) * (nj + 2) + (c % nj) + 1  # cell -> padded flat
        npad = (ni + 2) * (nj + 2)
        self.count = torch.tensor([len(c) for c in contrib], dtype=torch.float64, device=self.device)
        self.wall_r_base = torch.zeros(nn, dtype=torch.float64, device=self.device)
        mats = {}
        for comp in ("u", "v", "t", "rho", "r"):
            rows, cols = [], []
            last = resets.get(comp, [-1] * nn)
            for n in range(nn):
                for pos, (kind, idx) in enumerate(contrib[n]):
                    if pos <= last[n]:
                        continue
                    rows.append(n)
                    cols.append(cflat(idx) if kind == 0 else gflat[idx])
            mats[comp] = (torch.tensor(rows, dtype=torch.int64, device=self.device),
                          torch.tensor(cols, dtype=torch.int64, device=self.device))
        self.navg = mats
        self.r_reset = torch.tensor([1.0 if resets["r"][n] >= 0 else 0.0 for n in range(nn)],
                                    dtype=torch.float64, device=self.device)

    def time_step(self, C, geo, prm: Params):
        """turbnstwod.f90:97-114."""
        rho = C[0]
        u, v = C[1] / rho, C[2] / rho
        vel = torch.sqrt(u * u + v * v)
        t = (C[3] / rho - 0.5 * (u * u + v * v)) / prm.cv
        p = rho * prm.rr * t
        dt = self.flow.cfl * geo["dl"] / (torch.abs(vel) + torch.sqrt(self.flow.gama * prm.rr * t))
        if self.flow.local == 0:
            dt = torch.full_like(dt, 1.0) * torch.min(dmin(torch.full_like(dt, 100000.0), dt))
        return dt, p

    def dissipation(self, C, p, dt, geo, rtol):
        """DISSIPATION (solver_state.f90:70-225); ghosts hold copies of their parent.
        Returns D [5, NI, NJ]."""
        Pn = self._nb(_pad(p))
        anu = (torch.abs(Pn[0] - p) + torch.abs(Pn[1] - p) + torch.abs(Pn[2] - p) + torch.abs(Pn[3] - p)) / \
              (torch.abs(Pn[0] + p) + torch.abs(Pn[1] + p) + torch.abs(Pn[2] + p) + torch.abs(Pn[3] + p))
        Cp = _pad(C)
        Cn = self._nb(Cp)
        c5 = C[4]
        c5n = [x[4] for x in Cn]
        anurt = (torch.abs(c5n[0] - c5) + torch.abs(c5n[1] - c5) + torch.abs(c5n[2] - c5) +
                 torch.abs(c5n[3] - c5)) / dmax(torch.abs(c5n[0] + c5) + torch.abs(c5n[1] + c5) +
                                                torch.abs(c5n[2] + c5) + torch.abs(c5n[3] + c5),
                                                8.0 * C[0] * rtol)
        d2q = Cn[0] + Cn[1] + Cn[2] + Cn[3] - 4.0 * C
        dn = self._nb(_pad(d2q))
        vbd = geo["vol"] / dt
        vbdn = self._nb(_pad(vbd))
        S = _pad(torch.stack([anu, anurt]))
        si = S[:, 1:-1, 1:-1]
        sn = self._nb(S)
        comp = self.sensor_of  # sensor of each equation: ANU for 1-4, ANURT for 5
        D2 = D4 = None
        for k in range(4):
            e2 = C02 * dmax(si, sn[k])
            e4 = dmax(torch.zeros_like(e2), C04 - e2)
            d24 = 0.5 * (vbd + vbdn[k])
            t2 = (e2 * d24).index_select(0, comp) * (Cn[k] - C)
            t4 = (e4 * d24).index_select(0, comp) * (dn[k] - d2q)
            D2 = t2 if D2 is None else D2 + t2
            D4 = t4 if D4 is None else D4 + t4
        return D2 - D4

    def viscous(self, full, geo, prm: Params, rtol):
        """COMPUTE_VISCOUS (viscous.f90:29-217) from the padded field set of stage 1.
        Returns VIS [4, NI, NJ]."""
        flow = self.flow
        ni, nj = self.ni, self.nj
        rho = full[C_]
        vals = torch.stack([full[U_], full[V_], full[T_], rho, full[C_ + 4] / rho])  # u v t rho r
        flat = vals.reshape(5, -1)
        nodes = []
        for k, name in enumerate(("u", "v", "t", "rho", "r")):
            rows, cols = self.navg[name]
            sacc = torch.zeros(self.count.shape[0], dtype=vals.dtype, device=vals.device).index_add(
                0, rows, flat[k].index_select(0, cols))
            if name == "r":
                sacc = sacc + self.r_reset * (rtol * flow.rtred)
            nodes.append(sacc / self.count)
        nodes = torch.stack(nodes).reshape(5, ni + 1, nj + 1)
        nodes = torch.cat([nodes[:4], dmax(torch.zeros_like(nodes[4:]) + rtol, nodes[4:])])
        x, y = geo["x"], geo["y"]
        corner = [(slice(None, -1), slice(None, -1)), (slice(1, None), slice(None, -1)),
                  (slice(1, None), slice(1, None)), (slice(None, -1), slice(1, None))]
        A = vals[:, 1:-1, 1:-1]
        xa, ya = geo["xc"][1:-1, 1:-1], geo["yc"][1:-1, 1:-1]
        nbs = self._nb(vals)
        xcn, ycn = self._nb(geo["xc"]), self._nb(geo["yc"])
        amu_c = SUTH * math.sqrt(flow.amol)
        vis = None
        for face in range(4):
            b, d = corner[face], corner[(face + 1) % 4]
            XB, YB, XD, YD = x[b], y[b], x[d], y[d]
            B, D = nodes[(slice(None),) + b], nodes[(slice(None),) + d]
            Cc = nbs[face]
            XC, YC = xcn[face], ycn[face]
            dnr = (xa - XC) * (YB - YD) - (XB - XD) * (ya - YC)
            GX = ((A - Cc) * (YB - YD) - (B - D) * (ya - YC)) / dnr
            GY = (-(A - Cc) * (XB - XD) + (B - D) * (xa - XC)) / dnr
            DUX, DVX, DTX, DRX = GX[0], GX[1], GX[2], GX[4]
            DUY, DVY, DTY, DRY = GY[0], GY[1], GY[2], GY[4]
            AV = 0.25 * (A + B + Cc + D)
            UAVG, VAVG, TAVG, RHOAVG, RAVG = AV[0], AV[1], AV[2], AV[3], AV[4]
            if flow.iaxis == 1:
                YAVG = 0.5 * (YB + YD)
                near = YAVG < YAXIS_THRESH
                # the unselected branch divides by YAVG = 0 on axis faces: keep its
                # gradient finite (torch.where passes 0 * inf = NaN otherwise)
                VBYY = torch.where(near, DVY, VAVG / torch.where(near, torch.ones_like(YAVG), YAVG))
                DIVVEL = DUX + DVY + VBYY
            else:
                DIVVEL = DUX + DVY
            AMU = amu_c * TAVG ** 0.6
            AK = AMU * prm.cp / flow.prandtl
            CHI = RHOAVG * RAVG / (AMU * CMU)
            FMU = torch.tanh(ALPHA_T * CHI * CHI) / torch.tanh(BETA_T * CHI * CHI)
            AMUT = RHOAVG * RAVG * FMU
            AKT = AMUT * prm.cp / flow.prandtlt
            AMUEFF = AMU + AMUT
            AKEFF = AK + AKT
            div23 = 2.0 / 3.0
            TXX = AMUEFF * (DUX + DUX - div23 * DIVVEL)
            TYY = AMUEFF * (DVY + DVY - div23 * DIVVEL)
            TXY = AMUEFF * (DUY + DVX)
            QXX = UAVG * TXX + VAVG * TXY + AKEFF * DTX
            QYY = UAVG * TXY + VAVG * TYY + AKEFF * DTY
            SX, SY = geo["sx"][face], geo["sy"][face]
            f = torch.stack([TXX * SX + TXY * SY, TXY * SX + TYY * SY, QXX * SX + QYY * SY,
                             AMUEFF * DRX * SX + AMUEFF * DRY * SY])
            vis = f if vis is None else vis + f
        return vis

    def source(self, full, geo, prm: Params):
        """COMPUTE_SOURCE_TERMS (source_terms.f90:24-104): (SOURCE3, SOURCE5)."""
        flow = self.flow
        u, v = full[U_], full[V_]
        r = full[C_ + 4] / full[C_]
        q = torch.sqrt(u * u + v * v)
        stk = torch.stack([q, r, u, v])
        F = self._nb(stk)  # A, B, C, D = NC1..NC4
        X, Y = self._nb(geo["xc"]), self._nb(geo["yc"])
        XA, XB, XC, XD = X
        YA, YB, YC, YD = Y
        dnr = (XA - XC) * (YB - YD) - (XB - XD) * (YA - YC)
        GX = ((F[0] - F[2]) * (YB - YD) - (F[1] - F[3]) * (YA - YC)) / dnr
        GY = (-(F[0] - F[2]) * (XB - XD) + (F[1] - F[3]) * (XA - XC)) / dnr
        DQX, DRX, DUX, DVX = GX[0], GX[1], GX[2], GX[3]
        DQY, DRY, DUY, DVY = GY[0], GY[1], GY[2], GY[3]
        rho = full[C_][1:-1, 1:-1]
        ri = full[C_ + 4][1:-1, 1:-1] / rho
        amu = self.amu(full[T_][1:-1, 1:-1])
        chi = rho * ri / (CMU * amu)
        fmu = torch.tanh(ALPHA_T * chi * chi) / torch.tanh(BETA_T * chi * chi)
        fr2 = torch.tanh(torch.sqrt(chi)) / torch.tanh(chi * math.sqrt(2.0 * math.sqrt(CMU)))
        amut = fmu * rho * ri
        phi = DQX * DRX + DQY * DRY
        dee = torch.where(phi > 0.0, DRX * DRX + DRY * DRY, torch.zeros_like(phi))
        div23 = 2.0 / 3.0
        ycc = geo["yc"][1:-1, 1:-1]
        if flow.iaxis == 1:
            near = ycc < YAXIS_THRESH
            vbyy = torch.where(near, DVY, full[V_][1:-1, 1:-1] / torch.where(near, torch.ones_like(ycc), ycc))
            divvel = DUX + DVY + vbyy
            pk = amut / rho * (DUX * DUX + DVY * DVY + vbyy * vbyy + DUX * DUX + DVY * DVY +
                               vbyy * vbyy + (DUY + DVX) * (DUY + DVX) - div23 * divvel * divvel)
        else:
            divvel = DUX + DVY
            pk = amut / rho * (DUX * DUX + DVY * DVY + DUX * DUX + DVY * DVY +
                               (DUY + DVX) * (DUY + DVX) - div23 * divvel * divvel)
        pk = dmax(pk, torch.zeros_like(pk))
        ratio = amut / dmax(amut, AMU_THRESH * amu)
        pw = ratio ** flow.npseudo if flow.npseudo >= 0 else 1.0 / ratio ** (-flow.npseudo)
        s5 = (rho * (CONST1 - CONST2 * fr2) * _safe_sqrt(ri * pk) - rho * CONST3 * dee) * pw
        s3 = None
        if flow.iaxis == 1:
            ttt = (amu + amut) * (vbyy + vbyy - div23 * divvel)
            s3 = (full[P_][1:-1, 1:-1] - ttt) / ycc
        return s3, s5

    def residual(self, full, geo, s3, s5):
        """COMPUTE_RESIDUAL (residual.f90:23-62): R [5, NI, NJ]."""
        sx, sy = geo["sx"], geo["sy"]
        F, G = full[F_:F_ + 5], full[G_:G_ + 5]
        FI, GI = F[:, 1:-1, 1:-1], G[:, 1:-1, 1:-1]
        Fn, Gn = self._nb(F), self._nb(G)
        acc = (FI + Fn[0]) * sx[0] + (GI + Gn[0]) * sy[0]
        for k in range(1, 4):
            acc = acc + (FI + Fn[k]) * sx[k] + (GI + Gn[k]) * sy[k]
        R = 0.5 * acc
        r2 = R[2] - geo["vol"] * s3 if self.flow.iaxis == 1 else R[2]
        return torch.stack([R[0], R[1], r2, R[3], R[4] - geo["vol"] * s5])

    def iteration(self, Cold, geo, prm: Params):
        """One RK4 iteration (turbnstwod.f90:97-146): Q_old [5, NI, NJ] -> Q_new."""
        rtol = self.rtol(prm)
        dt, p = self.time_step(Cold, geo, prm)
        D = self.dissipation(Cold, p, dt, geo, rtol)
        C = Cold
        vis = None
        dtbyvol = dt / geo["vol"]
        for st in range(4):
            full = self.boundary(self.primitive(C, prm), prm, geo)
            if st == 0:
                vis = self.viscous(full, geo, prm, rtol)
                # the viscous terms of equations 2..5, none in the continuity equation
                vis5 = torch.cat([torch.zeros_like(vis[:1]), vis])
            s3, s5 = self.source(full, geo, prm)
            R = self.residual(full, geo, s3, s5)
            dtv = ALPHA_RK[st] * dtbyvol
            N = Cold - dtv * (R - vis5 - D)
            n4 = Cold[4] - dtv * CFLTURB * (R[4] - vis[3] - D[4])
            n0 = N[0]
            n4 = n0 * dmax(torch.zeros_like(n0) + rtol, n4 / n0)
            C = torch.cat([N[:4], n4[None]])
        return C


class GraphedStep:
    """The reverse step of one iteration -- recompute Q_{n+1} = G(Q_n, p) and pull
    lambda back: (lambda dG/dQ_n, lambda dG/dp) -- captured once as a CUDA graph with
    static input tensors and replayed for every n.  The step is a few thousand small
    kernels; replaying them from a graph removes the per-kernel launch cost of eager
    execution.  Results equal the eager step up to the summation order of index_add."""

    def __init__(self, scheme: Scheme, space: DesignSpace, params: List[torch.Tensor], dy_index: Optional[int]):
        self.scheme, self.space, self.dy_index = scheme, space, dy_index
        ni, nj = scheme.ni, scheme.nj
        z = dict(dtype=torch.float64, device=scheme.device)
        side = torch.cuda.Stream(device=scheme.device)
        side.wait_stream(torch.cuda.current_stream(scheme.device))
        with torch.cuda.stream(side):
            # leaves of its own, first used on the warm-up stream: autograd then never
            # synchronises with the stream the caller's leaves were first used on
            self.params = [p.detach().clone().requires_grad_(True) for p in params]
            self.Q = torch.zeros((5, ni, nj), **z).requires_grad_(True)
            self.lam = torch.zeros((5, ni, nj), **z)
            with torch.no_grad():  # a finite state for the warm-up steps
                self.Q.copy_(scheme.cold_state(self._prm()))
            for _ in range(2):
                self._step()
        torch.cuda.current_stream(scheme.device).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.out = self._step()

    def _prm(self):
        p = self.params
        return Params(p[0], p[1], p[2], self.scheme.flow)

    def _step(self):
        dy = self.params[self.dy_index] if self.dy_index is not None else None
        x, y = self.space.coords(dy)
        geo = self.scheme.geometry(x, y)
        Qn1 = self.scheme.iteration(self.Q, geo, self._prm())
        # lambda . G as a scalar: its gradient is the vector-Jacobian product, and the
        # seed of the backward pass is then created inside the capture
        g = torch.autograd.grad(torch.sum(Qn1 * self.lam), [self.Q] + self.params, allow_unused=True)
        return [v if v is not None else torch.zeros_like(p) for v, p in zip(g, [self.Q] + self.params)]

    def __call__(self, Qn: torch.Tensor, lam: torch.Tensor):
        with torch.no_grad():
            self.Q.copy_(Qn)
            self.lam.copy_(lam)
        self.graph.replay()
        return [t.clone() for t in self.out]


def transient_gradient_torch(scheme: Scheme, objective: Callable, p0=None, t0=None, amachinit=None,
                             dy: Optional[torch.Tensor] = None, space: Optional[DesignSpace] = None,
                             niter: int = 100, states: Optional[np.ndarray] = None, primal: str = "gpu",
                             lib=None, graph: Optional[bool] = None) -> dict:
    """The autograd reverse sweep: dJ/d(P0, T0, AMACHINIT, dy) of J = objective(scheme, Q_N,
    geo, prm), Q_0 the cold start.  The primal runs on the GPU FP64 path
    (``primal="gpu"``) or in the restatement (``"torch"``); ``states`` may pass
    precomputed checkpoints [N+1, 5, NELES].  The sweep recomputes each iteration from
    its checkpoint inside autograd; on a CUDA device that step is captured once as a
    CUDA graph (``graph``, default on)."""
    dev = scheme.device
    leaf = lambda v, d: torch.tensor(float(d if v is None else v), dtype=torch.float64, device=dev,
                                     requires_grad=True)
    P0, T0, AM = leaf(p0, scheme.flow.p0), leaf(t0, scheme.flow.t0), leaf(amachinit, scheme.flow.amachinit)
    if dy is not None:
        dy = dy.detach().clone().to(dev).requires_grad_(True)
    space = space or DesignSpace(scheme)
    ni, nj = scheme.ni, scheme.nj

    def setup():
        prm = Params(P0, T0, AM, scheme.flow)
        x, y = space.coords(dy)
        return prm, scheme.geometry(x, y)

    with torch.no_grad():
        prm, geo = setup()
        c0 = scheme.cold_state(prm)
    if states is None:
        if primal == "gpu":
            mesh_now = _mesh_with_coords(scheme, space, dy)
            f = dataclasses.replace(scheme.flow, p0=float(P0.detach()), t0=float(T0.detach()),
                                    amachinit=float(AM.detach()))
            rinit = float(scheme.rtol(prm).detach() / scheme.flow.rtred)
            states = primal_gpu(mesh_now, f, c0.reshape(5, -1).cpu().numpy(), rinit, niter, lib)
        else:
            with torch.no_grad():
                c, states = c0, [c0.reshape(5, -1).cpu().numpy()]
                for _ in range(niter):
                    c = scheme.iteration(c, geo, prm)
                    states.append(c.reshape(5, -1).cpu().numpy())
                states = np.stack(states)
    ck = lambda n: torch.tensor(states[n].reshape(5, ni, nj), dtype=torch.float64, device=dev)

    params = [P0, T0, AM] + ([dy] if dy is not None else [])
    grads = [torch.zeros_like(p) for p in params]

    def accumulate(g):
        for k, v in enumerate(g):
            if v is not None:
                grads[k] = grads[k] + v

    # dJ/dQ_N and the direct dependence of J on the parameters
    QN = ck(niter).requires_grad_(True)
    prm, geo = setup()
    J = objective(scheme, QN, geo, prm)
    g = torch.autograd.grad(J, [QN] + params, allow_unused=True)
    lam = g[0]
    accumulate(g[1:])
    # reverse sweep over the iterations
    if graph is None:
        graph = scheme.device.type == "cuda"
    step = GraphedStep(scheme, space, params, 3 if dy is not None else None) if graph and niter > 0 else None
    for n in range(niter - 1, -1, -1):
        if step is not None:
            g = step(ck(n), lam)
        else:
            Qn = ck(n).requires_grad_(True)
            prm, geo = setup()
            Qn1 = scheme.iteration(Qn, geo, prm)
            g = torch.autograd.grad(Qn1, [Qn] + params, grad_outputs=lam, allow_unused=True)
        lam = g[0]
        accumulate(g[1:])
    del step
    # the cold start Q_0(P0, T0, AMACHINIT)
    prm, geo = setup()
    Q0 = scheme.cold_state(prm)
    g = torch.autograd.grad(Q0, params, grad_outputs=lam, allow_unused=True)
    accumulate(g)
    out = {"J": float(J.detach()), "dJ_dp0": float(grads[0]), "dJ_dt0": float(grads[1]),
           "dJ_damachinit": float(grads[2]), "lambda0": lam.detach(), "states": states}
    if dy is not None:
        out["dJ_ddy"] = grads[3].detach().cpu().numpy()
    return out


def fixed_point_adjoint_torch(scheme: Scheme, objective: Callable, Qstar: torch.Tensor, niter: int = 200,
                              p0=None, t0=None, amachinit=None, dy=None, space=None) -> dict:
    """Autograd fixed-point adjoint at a steady state Q*: iterates lambda <- dJ/dQ +
    lambda dG/dQ and returns dJ/dp with the adjoint residual history."""
    dev = scheme.device
    leaf = lambda v, d: torch.tensor(float(d if v is None else v), dtype=torch.float64, device=dev,
                                     requires_grad=True)
    P0, T0, AM = leaf(p0, scheme.flow.p0), leaf(t0, scheme.flow.t0), leaf(amachinit, scheme.flow.amachinit)
    if dy is not None:
        dy = dy.detach().clone().to(dev).requires_grad_(True)
    space = space or DesignSpace(scheme)
    params = [P0, T0, AM] + ([dy] if dy is not None else [])
    prm = Params(P0, T0, AM, scheme.flow)
    x, y = space.coords(dy)
    geo = scheme.geometry(x, y)
    Q = Qstar.detach().clone().requires_grad_(True)
    J = objective(scheme, Q, geo, prm)
    gJ = torch.autograd.grad(J, [Q] + params, allow_unused=True, retain_graph=True)
    djdq = gJ[0]
    G = scheme.iteration(Q, geo, prm)
    lam = djdq.clone()
    hist = []
    for _ in range(niter):
        (vj,) = torch.autograd.grad(G, [Q], grad_outputs=lam, retain_graph=True)
        new = djdq + vj
        hist.append(float(torch.max(torch.abs(new - lam))))
        lam = new
    gp = torch.autograd.grad(G, params, grad_outputs=lam, allow_unused=True)
    grads = []
    for k, p in enumerate(params):
        v = torch.zeros_like(p)
        if gJ[k + 1] is not None:
            v = v + gJ[k + 1]
        if gp[k] is not None:
            v = v + gp[k]
        grads.append(v)
    out = {"J": float(J.detach()), "dJ_dp0": float(grads[0]), "dJ_dt0": float(grads[1]),
           "dJ_damachinit": float(grads[2]), "residual_history": hist, "lambda": lam.detach()}
    if dy is not None:
        out["dJ_ddy"] = grads[3].detach().cpu().numpy()
    return out

