"""Discrete adjoint (reverse-mode sensitivities) of the RK4 / JST / viscous scheme.

The reference has no adjoint.  This module gives gradients of an objective J(Q_N) of
the state after N RK4 iterations, or of a steady state, with respect to the inflow
parameters (P0, T0), the cold-start Mach number AMACHINIT and mesh-node coordinates
(wall shape).  The reverse steps are the hand-written CUDA adjoint of the C ABI
(csrc/tns_adjoint.*: tns_adjoint_step, tns_adjoint_record / tns_adjoint_step_recorded);
there is no other engine.

* ``Scheme`` holds what the gradient needs around those steps, as differentiable FP64
  tensor arithmetic on the structured i x j block: COMPUTE_GEOMETRY from the node
  coordinates (geometry.f90:55-149; node displacements are parameters), the parameter
  formulas (turbnstwod.f90:37-71), COMPUTE_PRIMITIVE_VARS (turbnstwod.f90:204-227) and
  APPLY_BOUNDARY for BC types 2-7 (boundary.f90:24-327), on which the objectives are
  evaluated.  The sensitivities the CUDA steps accumulate (face vectors, volumes, DL,
  centroids, node coordinates, RTOLERANCE, S0, T0) are mapped to the parameters by one
  torch backward through these formulas (``_parameter_gradient``).
* ``transient_gradient``: the primal on the GPU with a device checkpoint (or a record of
  the forward values) per iteration, then the reverse sweep of CUDA adjoint steps;
  ``max_states`` bounds the device memory with bisection snapshots.
  ``TransientObjective`` is the same as a ``torch.autograd.Function``.
* ``fixed_point_adjoint`` iterates lambda <- dJ/dQ + lambda dG/dQ with frozen forward
  values at a steady state, the adjoint of a converged solution.

Scope: IAXIS 0 and 1, BC types 2-7, any LOCAL and NPSEUDO.  Objective helpers evaluate
on the final state Q_N with its ghost cells from APPLY_BOUNDARY: the wall pressure
force and the mass-weighted total-pressure loss between two sides.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np
import torch

from .formats import Flow, Mesh

# constants.f90:12-60
RUNIV = 8314.0
CMU = 0.09
ALPHA_T = 0.00052
BETA_T = 0.2
CONST1 = 21.479
CONST2 = 21.394
CONST3 = 1.5
SUTH = 0.00000011848
C02 = 0.25
C04 = 0.00390625
CFLTURB = 0.5
YAXIS_THRESH = 0.001
AMU_THRESH = 0.001
ALPHA_RK = (0.25, 1.0 / 3.0, 0.5, 1.0)


def dmax(a, b):
    """DMAX1: a >= b ? a : b (gradient to the selected argument)."""
    return torch.where(a >= b, a, b)


def dmin(a, b):
    return torch.where(a <= b, a, b)


def _safe_sqrt(x):
    """sqrt with a zero gradient where x == 0 (PK clamped to 0 by DMAX1)."""
    pos = x > 0
    return torch.where(pos, torch.sqrt(torch.where(pos, x, torch.ones_like(x))), torch.zeros_like(x))


def _pad(a):
    """([k,] ni, nj) -> ([k,] ni+2, nj+2) with the ring holding copies of the adjacent
    cell."""
    if a.dim() == 2:
        return torch.nn.functional.pad(a[None, None], (1, 1, 1, 1), mode="replicate")[0, 0]
    return torch.nn.functional.pad(a[None], (1, 1, 1, 1), mode="replicate")[0]


# rows of the stacked primitive field set (COMPUTE_PRIMITIVE_VARS and the ghosts)
U_, V_, T_, P_ = 0, 1, 2, 3
C_, F_, G_ = 4, 9, 14     # C1..C5, F1..F5, G1..G5
NW_ = 19


@dataclasses.dataclass
class Params:
    """Flow parameters as tensors (P0, T0, AMACHINIT may carry gradients)."""
    p0: torch.Tensor
    t0: torch.Tensor
    amachinit: torch.Tensor
    flow: Flow

    @property
    def rr(self):
        return RUNIV / self.flow.amol

    @property
    def cv(self):
        return self.rr / (self.flow.gama - 1.0)

    @property
    def cp(self):
        return self.cv * self.flow.gama

    def s0(self):
        rho0 = self.p0 / (self.rr * self.t0)
        return self.p0 / rho0 ** self.flow.gama

    def cold(self):
        """Isentropic cold start (turbnstwod.f90:53-71): (RHO, U, E, RINIT)."""
        g = self.flow.gama
        dyn = 1.0 + (g - 1.0) * 0.5 * self.amachinit ** 2
        tinit = self.t0 / dyn
        pinit = self.p0 / dyn ** (g / (g - 1.0))
        uinit = self.amachinit * torch.sqrt(g * self.rr * tinit)
        einit = self.cv * tinit + 0.5 * uinit ** 2
        rhoinit = pinit / (self.rr * tinit)
        amu = SUTH * math.sqrt(self.flow.amol) * tinit ** 0.6
        return rhoinit, uinit, einit, amu / rhoinit


class Scheme:
    """Geometry, parameters, primitive variables, ghost states and objectives of one
    structured case as differentiable FP64 tensor arithmetic.

    ``mesh`` must be one structured block numbered as ``cases.structured_mesh`` numbers
    it (cell (i, j) id i*NJ+j+1, node (i, j) id i*(NJ+1)+j+1, faces 1..4 = j-, i+, j+,
    i-).  State tensors are [5, NI, NJ]; node coordinates [NI+1, NJ+1].
    """

    def __init__(self, mesh: Mesh, flow: Flow, device="cpu", rinit: Optional[float] = None):
        if mesh.shape is None:
            raise ValueError("the adjoint needs a structured block (Mesh.shape)")
        ni, nj = mesh.shape
        self.ni, self.nj, self.flow, self.device = ni, nj, flow, torch.device(device)
        ii, jj = np.meshgrid(np.arange(ni), np.arange(nj), indexing="ij")
        expect = np.stack([ii * (nj + 1) + jj + 1, (ii + 1) * (nj + 1) + jj + 1,
                           (ii + 1) * (nj + 1) + jj + 2, ii * (nj + 1) + jj + 2], -1).reshape(-1, 4)
        if not np.array_equal(mesh.nod, expect):
            raise ValueError("mesh is not in structured (i, j) numbering")
        if np.any((mesh.ntype < 2) | (mesh.ntype > 7)):
            bad = sorted(set(mesh.ntype.tolist()) - {2, 3, 4, 5, 6, 7})
            raise NotImplementedError(f"BC types {bad}: the adjoint covers types 2-7")
        if flow.iaxis not in (0, 1):
            raise ValueError("IAXIS must be 0 or 1")
        self.fixed_rinit = rinit
        self.mesh_template = mesh
        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        self.x0 = torch.tensor(mesh.x.reshape(ni + 1, nj + 1), **f64)
        self.y0 = torch.tensor(mesh.y.reshape(ni + 1, nj + 1), **f64)
        # BC type of each ghost, per side, along the side
        types = {1: np.zeros(ni, np.int64), 2: np.zeros(nj, np.int64), 3: np.zeros(ni, np.int64),
                 4: np.zeros(nj, np.int64)}
        par = mesh.nparent - 1
        pi, pj = par // nj, par % nj
        for k in range(mesh.nghosts):
            s = int(mesh.nside[k])
            types[s][pi[k] if s in (1, 3) else pj[k]] = mesh.ntype[k]
        self.types = {s: torch.tensor(v, device=dev) for s, v in types.items()}
        # every ghost of the ring at once: parent / opposite cell (flat interior index),
        # flat index in the padded field, BC type; sides 1, 3 along i, then 4, 2 along j
        ai, aj = np.arange(ni), np.arange(nj)
        par_i = np.concatenate([ai, ai, np.zeros(nj, int), np.full(nj, ni - 1)])
        par_j = np.concatenate([np.zeros(ni, int), np.full(ni, nj - 1), aj, aj])
        opp_i = np.concatenate([ai, ai, np.ones(nj, int), np.full(nj, ni - 2)])
        opp_j = np.concatenate([np.ones(ni, int), np.full(ni, nj - 2), aj, aj])
        g_i = np.concatenate([ai + 1, ai + 1, np.zeros(nj, int), np.full(nj, ni + 1)])
        g_j = np.concatenate([np.zeros(ni, int), np.full(ni, nj + 1), aj + 1, aj + 1])
        it = lambda a: torch.tensor(a, dtype=torch.int64, device=dev)
        self.g_par = it(par_i * nj + par_j)
        self.g_opp = it(opp_i * nj + opp_j)
        self.g_pad = it(g_i * (nj + 2) + g_j)
        self.g_type = torch.cat([self.types[1], self.types[3], self.types[4], self.types[2]])
        # type-6 burn-rate multiplier per ring ghost (bc.in order -> ring order)
        inj = np.ones(2 * (ni + nj))
        if mesh.inj_scale is not None:
            ring_off = {1: 0, 3: ni, 4: 2 * ni, 2: 2 * ni + nj}
            for k in range(mesh.nghosts):
                sd = int(mesh.nside[k])
                inj[ring_off[sd] + (pi[k] if sd in (1, 3) else pj[k])] = mesh.inj_scale[k]
        self.g_inj = torch.tensor(inj, dtype=torch.float64, device=dev)
        self.types_present = sorted(set(int(t) for t in np.unique(mesh.ntype)))
        self.sensor_of = torch.tensor([0, 0, 0, 0, 1], dtype=torch.int64, device=dev)

    # ------------------------------------------------------------------ set-up
    # ------------------------------------------------------------------ pieces
    def params(self, p0=None, t0=None, amachinit=None) -> Params:
        f = self.flow
        t = lambda v, d: torch.as_tensor(d if v is None else v, dtype=torch.float64, device=self.device)
        return Params(t(p0, f.p0), t(t0, f.t0), t(amachinit, f.amachinit), f)

    def rtol(self, prm: Params):
        rinit = self.fixed_rinit if self.fixed_rinit is not None else prm.cold()[3]
        return rinit * self.flow.rtred

    def cold_state(self, prm: Params):
        rho, u, e, rinit = prm.cold()
        if self.fixed_rinit is not None:
            rinit = self.fixed_rinit
        one = torch.ones((self.ni, self.nj), dtype=torch.float64, device=self.device)
        return torch.stack([rho * one, rho * u * one, 0.0 * one, rho * e * one, rho * rinit * one])

    def geometry(self, x, y) -> Dict[str, torch.Tensor]:
        """COMPUTE_GEOMETRY (geometry.f90:55-149) from node coordinates [NI+1, NJ+1]."""
        X1, X2, X3, X4 = x[:-1, :-1], x[1:, :-1], x[1:, 1:], x[:-1, 1:]
        Y1, Y2, Y3, Y4 = y[:-1, :-1], y[1:, :-1], y[1:, 1:], y[:-1, 1:]
        xcc = (X1 + X2 + X3 + X4) * 0.25
        ycc = (Y1 + Y2 + Y3 + Y4) * 0.25
        L = lambda xa, ya, xb, yb: torch.sqrt((xa - xb) * (xa - xb) + (ya - yb) * (ya - yb))
        dl = dmin(dmin(dmin(L(X1, Y1, X2, Y2), L(X2, Y2, X3, Y3)), L(X3, Y3, X4, Y4)), L(X4, Y4, X1, Y1))
        pts = [(X1, Y1), (X2, Y2), (X3, Y3), (X4, Y4)]
        sx, sy = [], []
        for k in range(4):
            (xa, ya), (xb, yb) = pts[k], pts[(k + 1) % 4]
            if self.flow.iaxis == 1:
                sx.append((yb - ya) * (ya + yb) * 0.5)
                sy.append(-(xb - xa) * (ya + yb) * 0.5)
            else:
                sx.append(yb - ya)
                sy.append(-(xb - xa))
        vol = 0.5 * ((X3 - X1) * (Y4 - Y2) - (X4 - X2) * (Y3 - Y1))
        if self.flow.iaxis == 1:
            vol = vol * ycc
        vol = torch.abs(vol)
        # mirrored ghost centroids: 2 * face midpoint - parent centroid
        xg, yg = _pad(xcc), _pad(ycc)
        xg = xg.clone()
        yg = yg.clone()
        xg[1:-1, 0] = 2.0 * (0.5 * (X1[:, 0] + X2[:, 0])) - xcc[:, 0]
        yg[1:-1, 0] = 2.0 * (0.5 * (Y1[:, 0] + Y2[:, 0])) - ycc[:, 0]
        xg[-1, 1:-1] = 2.0 * (0.5 * (X2[-1, :] + X3[-1, :])) - xcc[-1, :]
        yg[-1, 1:-1] = 2.0 * (0.5 * (Y2[-1, :] + Y3[-1, :])) - ycc[-1, :]
        xg[1:-1, -1] = 2.0 * (0.5 * (X3[:, -1] + X4[:, -1])) - xcc[:, -1]
        yg[1:-1, -1] = 2.0 * (0.5 * (Y3[:, -1] + Y4[:, -1])) - ycc[:, -1]
        xg[0, 1:-1] = 2.0 * (0.5 * (X4[0, :] + X1[0, :])) - xcc[0, :]
        yg[0, 1:-1] = 2.0 * (0.5 * (Y4[0, :] + Y1[0, :])) - ycc[0, :]
        return dict(x=x, y=y, xc=xg, yc=yg, dl=dl, vol=vol, sx=sx, sy=sy)

    def amu(self, t):
        return SUTH * math.sqrt(self.flow.amol) * t ** 0.6

    def primitive(self, C, prm: Params):
        """COMPUTE_PRIMITIVE_VARS (turbnstwod.f90:204-227) on the cells, as one stacked
        field set [19, NI, NJ]: U, V, T, P, C1..C5, F1..F5, G1..G5."""
        rho = C[0]
        u = C[1] / rho
        v = C[2] / rho
        e = C[3] / rho
        t = (e - 0.5 * (u * u + v * v)) / prm.cv
        p = rho * prm.rr * t
        rt = C[4] / rho
        f2 = rho * u * v
        return torch.stack([u, v, t, p, C[0], C[1], C[2], C[3], C[4],
                            C[1], rho * u * u + p, f2, (C[3] + p) * u, rho * rt * u,
                            C[2], f2, rho * v * v + p, (C[3] + p) * v, rho * rt * v])

    def _ghosts(self, pr, opp, prm: Params, ycg=None, port=None):
        """APPLY_BOUNDARY (boundary.f90:53-122, 310-327) for every ghost of the ring at
        once: parent field set ``pr`` [19, NG] and U, V, T, P of the cell opposite the
        boundary face ``opp`` [4, NG]; ``ycg`` [NG] the ghosts' mirrored centroid y
        (types 6, 7); ``port`` the type-6 inputs per ring ghost (port mass flux, the
        parent's face vector on the ghost side, the parent's centroid y).  Each BC type
        present in the mesh is evaluated on the whole ring and selected by the ghost's
        type."""
        flow = self.flow
        rr, cv, cp, g = prm.rr, prm.cv, prm.cp, flow.gama

        def state(rho, u, v, t, p, c5, f5, g5):
            c1, c2 = rho * u, rho * v
            c3 = rho * (cv * t + 0.5 * (u * u + v * v))
            f3 = rho * u * v
            return torch.stack([u, v, t, p, rho, c1, c2, c3, c5,
                                c1, rho * u * u + p, f3, (c3 + p) * u, f5,
                                c2, f3, rho * v * v + p, (c3 + p) * v, g5])

        sel = {}
        if 2 in self.types_present:  # subsonic inlet at P0, T0 (isentropic)
            u2 = torch.abs(pr[U_])
            v2 = -pr[V_]
            t2 = prm.t0 - 0.5 * (u2 * u2 + v2 * v2) / cp
            rho2 = (prm.s0() / (rr * t2)) ** (1.0 / (1.0 - g))
            p2 = rho2 * rr * t2
            c5 = rho2 * (self.amu(t2) / rho2)
            sel[2] = state(rho2, u2, v2, t2, p2, c5, c5 * u2, c5 * v2)
        if 3 in self.types_present:  # extrapolation (PAMB >= 0 fixes P)
            u3 = torch.abs(2.0 * pr[U_] - opp[0])
            v3 = 2.0 * pr[V_] - opp[1]
            t3 = 2.0 * pr[T_] - opp[2]
            p3 = 2.0 * pr[P_] - opp[3]
            if flow.pamb >= 0.0:
                p3 = torch.full_like(p3, flow.pamb)
            sel[3] = state(p3 / (rr * t3), u3, v3, t3, p3, pr[C_ + 4], pr[F_ + 4], pr[G_ + 4])
        if 4 in self.types_present:  # symmetry
            sel[4] = state(pr[C_], pr[U_], -pr[V_], pr[T_], pr[P_], pr[C_ + 4], pr[F_ + 4], -pr[G_ + 4])
        if 5 in self.types_present:  # no-slip wall
            u5, v5, rho5 = -pr[U_], -pr[V_], pr[C_]
            e5 = cv * pr[T_] + 0.5 * (u5 * u5 + v5 * v5)
            P = pr[P_]
            sel[5] = torch.stack([u5, v5, pr[T_], P, rho5, rho5 * u5, rho5 * v5, rho5 * e5, -pr[C_ + 4],
                                  -pr[F_], 2.0 * P - pr[F_ + 1], -pr[F_ + 2], -pr[F_ + 3], -pr[F_ + 4],
                                  -pr[G_], -pr[G_ + 1], 2.0 * P - pr[G_ + 2], -pr[G_ + 3], -pr[G_ + 4]])
        if 6 in self.types_present:  # mass injection (boundary.f90:128-163)
            gport, psx, psy, ycp = port
            six = self.g_type == 6
            # the other ghosts of the ring get harmless inputs (on an axis the face vector
            # and DHYD are 0): no NaN may reach the gradient through the unselected branch
            psx = torch.where(six, psx, torch.ones_like(psx))
            psy = torch.where(six, psy, torch.zeros_like(psy))
            gport = torch.where(six, gport, torch.zeros_like(gport))
            dnr = torch.sqrt(psx * psx + psy * psy)
            enx, eny = -psx / dnr, -psy / dnr
            dhyd = torch.abs(torch.where(six, ycg + ycp, torch.ones_like(ycg)))
            gp = 2.0 * gport / (dhyd * dhyd) if flow.iaxis == 1 else gport / dhyd
            rho0, p6 = pr[C_], pr[P_]
            rdot = flow.acomb * (p6 * (1.0 / 98066.5)) ** flow.ancomb * self.g_inj
            vel = flow.rhoprop / rho0 * rdot
            u1 = vel * enx + vel * enx - pr[U_]
            v1 = vel * eny + vel * eny - pr[V_]
            t1 = flow.tflame - 0.5 * (u1 * u1 + v1 * v1) / cp
            gval = (gp / (flow.rhoprop * rdot)) * (flow.rhoprop * rdot * dhyd / self.amu(t1)) ** (-0.125)
            ero = gval > 35.0  # GTH
            gsafe = torch.where(ero, gval, torch.full_like(gval, 35.0))
            rdoteb = torch.where(ero, rdot * (1.0 + 0.023 * (gsafe ** 0.8 - 35.0 ** 0.8)), rdot)
            vel = flow.rhoprop / rho0 * rdoteb
            u6 = vel * enx + vel * enx - pr[U_]
            v6 = vel * eny + vel * eny - pr[V_]
            t6 = flow.tflame - 0.5 * (u6 * u6 + v6 * v6) / cp
            rho6 = p6 / (rr * t6)
            c5 = rho6 * (self.amu(t6) / rho6)
            sel[6] = state(rho6, u6, v6, t6, p6, c5, c5 * u6, c5 * v6)
        if 7 in self.types_present:  # boundary-layer inlet, 1/7-power profile (boundary.f90:310-327)
            tinf = prm.t0 / (1.0 + 0.5 * (g - 1.0) * flow.aminf ** 2)
            blu = 2.0 * flow.aminf * torch.sqrt(g * rr * tinf)
            inside = ycg <= flow.deltabl
            # the profile is evaluated on the whole ring: keep the other ghosts (mirrored
            # below a wall, y < 0) out of the power so that no NaN gradient leaks
            ratio = torch.where(inside & (ycg > 0), ycg, torch.full_like(ycg, flow.deltabl)) / flow.deltabl
            u7 = torch.where(inside, blu * ratio ** (1.0 / 7.0), blu * torch.ones_like(ycg)) - pr[U_]
            v7 = -pr[V_]
            t7 = tinf * torch.ones_like(ycg)
            p7 = torch.full_like(ycg, flow.pinf)
            rho7 = p7 / (rr * t7)
            c5 = rho7 * (self.amu(t7) / rho7)
            sel[7] = state(rho7, u7, v7, t7, p7, c5, c5 * u7, c5 * v7)
        order = list(sel)
        out = sel[order[0]]
        for ty in order[1:]:
            out = torch.where(self.g_type == ty, sel[ty], out)
        return out

    def boundary(self, W, prm: Params, geo=None):
        """Padded field set [19, NI+2, NJ+2]: cells plus the ghosts of APPLY_BOUNDARY
        (type 7 reads the ghosts' centroids from ``geo``)."""
        flat = W.reshape(NW_, -1)
        pr = flat.index_select(1, self.g_par)
        opp = flat[:4].index_select(1, self.g_opp)
        ycg = port = None
        if 6 in self.types_present or 7 in self.types_present:
            if geo is None:
                raise ValueError("BC types 6 and 7 need the geometry")
            ycg = geo["yc"].reshape(-1).index_select(0, self.g_pad)
        if 6 in self.types_present:
            port = self._port_inputs(W, geo)
        gh = self._ghosts(pr, opp, prm, ycg, port)
        npad = (self.ni + 2) * (self.nj + 2)
        ring = torch.zeros((NW_, npad), dtype=W.dtype, device=W.device).index_copy(1, self.g_pad, gh)
        return torch.nn.functional.pad(W, (1, 1, 1, 1)) + ring.reshape(NW_, self.ni + 2, self.nj + 2)

    def _port_inputs(self, W, geo):
        """Type-6 inputs per ring ghost: the port mass flux GPORT, the sum over the
        cells of the ghost's line (the parent's column across to the opposite side) of
        C1 * U * DELY (* YCC for IAXIS=1), DELY the cell's extent normal to the ghost's
        side from its node y; and the parent's face vector and centroid y."""
        y = geo["y"]
        Y1, Y2, Y3, Y4 = y[:-1, :-1], y[1:, :-1], y[1:, 1:], y[:-1, 1:]
        c1 = W[C_]
        term = c1 * (W[C_ + 1] / c1)
        if self.flow.iaxis == 1:
            term = term * ((Y1 + Y2 + Y3 + Y4) * 0.25)
        g1 = torch.sum(term * (0.5 * ((Y1 + Y2) - (Y3 + Y4))), dim=1)
        g3 = torch.sum(term * (0.5 * ((Y3 + Y4) - (Y1 + Y2))), dim=1)
        g4 = torch.sum(term * (0.5 * ((Y4 + Y1) - (Y2 + Y3))), dim=0)
        g2 = torch.sum(term * (0.5 * ((Y2 + Y3) - (Y1 + Y4))), dim=0)
        gport = torch.cat([g1, g3, g4, g2])
        sx, sy = geo["sx"], geo["sy"]
        psx = torch.cat([sx[0][:, 0], sx[2][:, -1], sx[3][0, :], sx[1][-1, :]])
        psy = torch.cat([sy[0][:, 0], sy[2][:, -1], sy[3][0, :], sy[1][-1, :]])
        ycp = geo["yc"][1:-1, 1:-1].reshape(-1).index_select(0, self.g_par)
        return gport, psx, psy, ycp

    # ------------------------------------------------------------------ objectives
    def face_state(self, C, prm: Params, side: int, geo=None):
        """Face values (parent + ghost)/2 on one side of the final state: U, V, P, RHO, T
        (RHO = P/(RR*T) on both sides of the face) and the face vector S."""
        full = self.boundary(self.primitive(C, prm), prm, geo)
        idx = {1: ((slice(1, -1), 1), (slice(1, -1), 0)), 3: ((slice(1, -1), -2), (slice(1, -1), -1)),
               4: ((1, slice(1, -1)), (0, slice(1, -1))), 2: ((-2, slice(1, -1)), (-1, slice(1, -1)))}[side]
        pa, gh = idx
        avg = lambda a: 0.5 * (a[pa] + a[gh])
        rho = full[P_] / (prm.rr * full[T_])
        return {"u": avg(full[U_]), "v": avg(full[V_]), "p": avg(full[P_]), "rho": avg(rho),
                "t": avg(full[T_])}

    def side_vectors(self, geo, side: int):
        face = side - 1
        sl = {1: (slice(None), 0), 3: (slice(None), -1), 4: (0, slice(None)), 2: (-1, slice(None))}[side]
        return geo["sx"][face][sl], geo["sy"][face][sl]

    def wall_force(self, C, geo, prm: Params, side: int = 1):
        """Pressure force sum(p_f S) over the faces of ``side`` (per radian when IAXIS=1)."""
        fs = self.face_state(C, prm, side, geo)
        sx, sy = self.side_vectors(geo, side)
        return torch.stack([torch.sum(fs["p"] * sx), torch.sum(fs["p"] * sy)])

    def total_pressure_loss(self, C, geo, prm: Params, inlet: int = 4, outlet: int = 2):
        """1 - mass-weighted outlet P0 / mass-weighted inlet P0."""
        g = self.flow.gama

        def mean(side):
            fs = self.face_state(C, prm, side, geo)
            sx, sy = self.side_vectors(geo, side)
            m2 = (fs["u"] ** 2 + fs["v"] ** 2) / (g * prm.rr * fs["t"])
            p0 = fs["p"] * (1.0 + 0.5 * (g - 1.0) * m2) ** (g / (g - 1.0))
            md = torch.abs(fs["rho"] * (fs["u"] * sx + fs["v"] * sy))
            return torch.sum(p0 * md) / torch.sum(md)

        return 1.0 - mean(outlet) / mean(inlet)


# ---------------------------------------------------------------------- parameters

@dataclasses.dataclass
class DesignSpace:
    """Parameters of a gradient: P0, T0, AMACHINIT and displacements of chosen nodes.

    ``node_ids`` are 0-based flat node indices (i*(NJ+1)+j); ``node_shape`` [n, NI+1,
    NJ+1] gives how each displacement moves every node's y (for a wall node blended to
    zero at the opposite boundary, the generator's (1 - f_j) column)."""
    scheme: Scheme
    node_shape: Optional[torch.Tensor] = None  # [n, NI+1, NJ+1]

    def coords(self, dy: Optional[torch.Tensor]):
        s = self.scheme
        if dy is None or self.node_shape is None:
            return s.x0, s.y0
        return s.x0, s.y0 + torch.einsum("k,kij->ij", dy.to(self.node_shape.device), self.node_shape)


def ramp_wall_shape(scheme: Scheme, wall_nodes: Sequence[int], blend: np.ndarray) -> torch.Tensor:
    """Unit displacement fields for ramp-wall nodes i in ``wall_nodes``: node (i, j)
    moves by blend[j] (``cases.ramp_mesh`` blends a wall displacement linearly to zero
    at the top: 1 - f_j)."""
    ni, nj = scheme.ni, scheme.nj
    out = torch.zeros((len(wall_nodes), ni + 1, nj + 1), dtype=torch.float64, device=scheme.device)
    for k, i in enumerate(wall_nodes):
        out[k, i, :] = torch.as_tensor(blend, dtype=torch.float64, device=scheme.device)
    return out


# ---------------------------------------------------------------------- gradients

def _objective_value(scheme, objective, C, geo, prm):
    return objective(scheme, C, geo, prm)


def primal_gpu(mesh: Mesh, flow: Flow, c0: np.ndarray, rinit: float, niter: int, lib=None):
    """The primal on the GPU through the C ABI (FP64): states Q_0 .. Q_N as [N+1, 5, NELES]."""
    from .solver import Solver
    s = Solver(mesh, flow, rinit, precision=0, lib=lib)
    try:
        s.upload(c0)
        states = [np.array(c0)]
        for _ in range(niter):
            s.run(1, 0)
            states.append(s.download())
        return np.stack(states)
    finally:
        s.close()


def transient_gradient(scheme: Scheme, objective: Callable, p0=None, t0=None, amachinit=None,
                       dy: Optional[torch.Tensor] = None, space: Optional[DesignSpace] = None,
                       niter: int = 100, states: Optional[np.ndarray] = None, lib=None,
                       max_states: Optional[int] = None, record: Optional[bool] = None) -> dict:
    """dJ/d(P0, T0, AMACHINIT, dy) of J = objective(scheme, Q_N, geo, prm), Q_0 the cold
    start, Q_N after ``niter`` RK4 iterations.

    The primal runs on the GPU FP64 path keeping a device checkpoint per iteration, and
    every reverse step is the hand-written CUDA adjoint of the C ABI (tns_adjoint_step),
    which also accumulates the sensitivities to geometry, RTOLERANCE, S0 and T0; one
    torch backward through COMPUTE_GEOMETRY and the parameter formulas maps those to the
    gradient.  ``states`` (optional) are checkpoints [N+1, 5, NI, NJ]; the result's
    "states" is the device tensor of checkpoints.  ``max_states`` bounds the device
    states held at once: the sweep then keeps snapshots at recursive bisection points and
    recomputes each segment's states from its snapshot (O(N log2(N / max_states)) extra
    primal iterations, the same gradient bit for bit; "states" is then None).  ``record``
    keeps every iteration's forward values from the primal (tns_adjoint_record, about 25
    doubles a cell an iteration) so that the reverse steps need not recompute them;
    default: when they fit in half the free device memory.  Needs a Scheme on a CUDA
    device."""
    return _transient_gradient_cuda(scheme, objective, p0, t0, amachinit, dy, space, niter, states, lib,
                                    max_states, record)


def _mesh_with_coords(scheme: Scheme, space: DesignSpace, dy) -> Mesh:
    """A formats.Mesh for the C ABI with the displaced node coordinates."""
    from . import cases
    x, y = space.coords(dy.detach() if dy is not None else None)
    m = scheme.mesh_template
    return dataclasses.replace(m, x=x.detach().cpu().numpy().ravel().copy(),
                               y=y.detach().cpu().numpy().ravel().copy(), x_mm=None, y_mm=None)


def objective_gpu(scheme: Scheme, objective: Callable, p0=None, t0=None, amachinit=None, dy=None,
                  space: Optional[DesignSpace] = None, niter: int = 100, lib=None) -> float:
    """J after ``niter`` iterations of the GPU FP64 primal from the cold start, for the
    given parameters (the evaluation central differences use)."""
    from .solver import Solver
    dev = scheme.device
    t = lambda v, d: torch.tensor(float(d if v is None else v), dtype=torch.float64, device=dev)
    prm = Params(t(p0, scheme.flow.p0), t(t0, scheme.flow.t0), t(amachinit, scheme.flow.amachinit),
                 scheme.flow)
    space = space or DesignSpace(scheme)
    with torch.no_grad():
        dyt = None if dy is None else torch.as_tensor(dy, dtype=torch.float64, device=dev)
        c0 = scheme.cold_state(prm).reshape(5, -1).cpu().numpy()
        mesh_now = _mesh_with_coords(scheme, space, dyt)
        f = dataclasses.replace(scheme.flow, p0=float(prm.p0), t0=float(prm.t0),
                                amachinit=float(prm.amachinit))
        s = Solver(mesh_now, f, float(scheme.rtol(prm).detach() / scheme.flow.rtred), precision=0, lib=lib)
        try:
            s.upload(c0)
            if niter:
                s.run(niter, 0)
            q = s.download()
        finally:
            s.close()
        x, y = space.coords(dyt)
        geo = scheme.geometry(x, y)
        C = torch.tensor(q.reshape(5, scheme.ni, scheme.nj), dtype=torch.float64, device=dev)
        return float(objective(scheme, C, geo, prm))


def fixed_point_adjoint(scheme: Scheme, objective: Callable, Qstar: torch.Tensor, niter: int = 200,
                        p0=None, t0=None, amachinit=None, dy=None, space=None, lib=None,
                        history_every: int = 1) -> dict:
    """Adjoint of a steady state Q* = G(Q*, p): iterates lambda <- dJ/dQ + lambda dG/dQ
    (the RK4 iteration's transposed Jacobian at Q*, tns_adjoint_step on frozen forward
    values) and returns dJ/dp = dJ/dp|direct + lambda dG/dp, with the adjoint residual
    history |lambda_{k+1} - lambda_k|_max recorded every ``history_every`` sweeps.
    Meaningful when Q* is a converged state of the primal.  Needs a Scheme on a CUDA
    device."""
    return _fixed_point_cuda(scheme, objective, Qstar, niter, p0, t0, amachinit, dy, space, lib,
                             history_every)


# ---------------------------------------------------------------------- CUDA engine

SENS_ORDER = ("sx", "sy", "vol", "dl", "xc", "yc", "x", "y", "rtolc", "rtoln", "t0", "s0")


def split_sensitivities(sens: np.ndarray, ni: int, nj: int, device) -> Dict[str, torch.Tensor]:
    """The accumulated sensitivities of tns_adjoint_sensitivities as the entries of
    ``Scheme.geometry`` (sx, sy lists of 4; vol, dl [NI, NJ]; xc, yc [NI+2, NJ+2]; x, y
    [NI+1, NJ+1]) and the scalars rtol, t0, s0."""
    n, npad, nnode = ni * nj, (ni + 2) * (nj + 2), (ni + 1) * (nj + 1)
    size = {"sx": 4 * n, "sy": 4 * n, "vol": n, "dl": n, "xc": npad, "yc": npad, "x": nnode, "y": nnode,
            "rtolc": n, "rtoln": nnode, "t0": n, "s0": n}
    t = torch.tensor(sens, dtype=torch.float64, device=device)
    raw, o = {}, 0
    for k in SENS_ORDER:
        raw[k] = t[o:o + size[k]]
        o += size[k]
    return {"sx": [raw["sx"][k * n:(k + 1) * n].reshape(ni, nj) for k in range(4)],
            "sy": [raw["sy"][k * n:(k + 1) * n].reshape(ni, nj) for k in range(4)],
            "vol": raw["vol"].reshape(ni, nj), "dl": raw["dl"].reshape(ni, nj),
            "xc": raw["xc"].reshape(ni + 2, nj + 2), "yc": raw["yc"].reshape(ni + 2, nj + 2),
            "x": raw["x"].reshape(ni + 1, nj + 1), "y": raw["y"].reshape(ni + 1, nj + 1),
            "rtol": raw["rtolc"].sum() + raw["rtoln"].sum(), "t0": raw["t0"].sum(), "s0": raw["s0"].sum()}


class DeviceAdjoint:
    """The hand-written CUDA discrete adjoint of one case (C ABI tns_adjoint_*): an FP64
    handle for the mesh at the design point.  ``primal`` records device checkpoints
    Q_0..Q_N; ``step`` pulls lambda back through one iteration in place;
    ``sensitivities`` returns (and clears) the accumulated lambda dG/dp.

    The handle runs on a stream of its own (``stream``; the graph-captured step cannot
    run on the legacy default stream), ordered after torch's current stream on entry to
    each call and before it on exit, so callers use the tensors as usual."""

    def __init__(self, scheme: Scheme, space: DesignSpace, prm: Params, dy, lib=None):
        from .solver import Solver
        self.scheme = scheme
        with torch.no_grad():
            mesh_now = _mesh_with_coords(scheme, space, dy)
            f = dataclasses.replace(scheme.flow, p0=float(prm.p0), t0=float(prm.t0),
                                    amachinit=float(prm.amachinit))
            rinit = float(scheme.rtol(prm) / scheme.flow.rtred)
        self.solver = Solver(mesh_now, f, rinit, precision=0, lib=lib)
        self.stream = torch.cuda.Stream(device=scheme.device)
        self.solver.set_stream(self.stream.cuda_stream)
        self.solver._check(self.solver.L.tns_adjoint_enable(self.solver.h))

    def _enter(self):
        self.stream.wait_stream(torch.cuda.current_stream(self.scheme.device))

    def _leave(self):
        torch.cuda.current_stream(self.scheme.device).wait_stream(self.stream)

    def primal(self, c0: torch.Tensor, niter: int) -> torch.Tensor:
        """Checkpoints [niter+1, 5, NI, NJ] on the device from Q_0 = c0."""
        states = torch.empty((niter + 1,) + tuple(c0.shape), dtype=torch.float64, device=self.scheme.device)
        states[0].copy_(c0)
        self._enter()
        self.solver.state_from_device(states[0].data_ptr())
        for n in range(niter):
            self.solver.enqueue(1)
            self.solver.state_to_device(states[n + 1].data_ptr())
        self.solver.synchronize()
        self._leave()
        return states

    def primal_recorded(self, c0: torch.Tensor, niter: int):
        """Checkpoints [niter+1, 5, NI, NJ] and the iterations' forward values
        [niter, record size] (tns_adjoint_record), from Q_0 = c0."""
        states = torch.empty((niter + 1,) + tuple(c0.shape), dtype=torch.float64, device=self.scheme.device)
        recs = torch.empty((niter, self.solver.adjoint_record_size()), dtype=torch.float64,
                           device=self.scheme.device)
        states[0].copy_(c0)
        self._enter()
        for n in range(niter):
            self.solver.adjoint_record(states[n].data_ptr(), states[n + 1].data_ptr(), recs[n].data_ptr())
        self.solver.synchronize()
        self._leave()
        return states, recs

    def step(self, q: torch.Tensor, lam: torch.Tensor, sensitivities, frozen: bool = False,
             q_next: Optional[torch.Tensor] = None, rec: Optional[torch.Tensor] = None):
        """``sensitivities``: True (all), "scalars" (RTOLERANCE, T0, S0) or False.
        ``frozen``: q is the previous step's state (its forward values are reused).
        ``q_next``: the state of the next step, whose forward values are computed beside
        this reverse (it must stay unchanged until that step).  ``rec``: the iteration's
        recorded forward values (``primal_recorded``), used instead of recomputing."""
        for t in (q, lam) + tuple(x for x in (q_next, rec) if x is not None):
            if not (t.is_contiguous() and t.dtype == torch.float64):
                raise ValueError("q, q_next, rec and lambda must be contiguous float64 device tensors")
        self._enter()
        self.solver.adjoint_step(q.data_ptr(), lam.data_ptr(), sensitivities, frozen,
                                 q_next.data_ptr() if q_next is not None else None,
                                 rec.data_ptr() if rec is not None else None)
        self._leave()

    def sensitivities(self) -> Dict[str, torch.Tensor]:
        s = self.solver.adjoint_sensitivities(reset=True)
        return split_sensitivities(s, self.scheme.ni, self.scheme.nj, self.scheme.device)

    def close(self):
        self.solver.close()


def _parameter_gradient(scheme: Scheme, space: DesignSpace, params: List[torch.Tensor], dy,
                        sens: Dict[str, torch.Tensor], lam0: Optional[torch.Tensor]) -> List[torch.Tensor]:
    """lambda dG/dp summed over the reverse steps (``sens``) plus lambda_0 dQ_0/dp, mapped
    to the parameters by one backward through COMPUTE_GEOMETRY, RTOLERANCE(P0, T0,
    AMACHINIT), S0(P0, T0) and the cold start."""
    prm = Params(params[0], params[1], params[2], scheme.flow)
    x, y = space.coords(dy)
    geo = scheme.geometry(x, y)
    outs, gos = [], []

    def add(t, g):
        if isinstance(t, torch.Tensor) and t.requires_grad:
            outs.append(t)
            gos.append(g)

    for k in ("x", "y", "xc", "yc", "dl", "vol"):
        add(geo[k], sens[k])
    for k in range(4):
        add(geo["sx"][k], sens["sx"][k])
        add(geo["sy"][k], sens["sy"][k])
    add(scheme.rtol(prm), sens["rtol"])
    add(prm.s0(), sens["s0"])
    add(prm.t0, sens["t0"])
    if lam0 is not None:
        add(scheme.cold_state(prm), lam0)
    g = torch.autograd.grad(outs, params, grad_outputs=gos, allow_unused=True)
    return [v if v is not None else torch.zeros_like(p) for v, p in zip(g, params)]


def _leaves(scheme, p0, t0, amachinit, dy):
    dev = scheme.device
    leaf = lambda v, d: torch.tensor(float(d if v is None else v), dtype=torch.float64, device=dev,
                                     requires_grad=True)
    P0, T0, AM = leaf(p0, scheme.flow.p0), leaf(t0, scheme.flow.t0), leaf(amachinit, scheme.flow.amachinit)
    if dy is not None:
        dy = dy.detach().clone().to(dev).requires_grad_(True)
    return [P0, T0, AM] + ([dy] if dy is not None else []), dy


class _Checkpoints:
    """Bounded device memory for the reverse sweep: ``cap`` state slots.  ``sweep(lo,
    hi, slot)`` runs the reverse steps hi-1 .. lo from the state at iteration lo (held in
    ``slot``).  If the segment's states fit in the free slots, they are recomputed and
    stored, then reversed; with one free slot left, each state is recomputed from the
    snapshot in turn; otherwise the state at the midpoint is recomputed into a slot, the
    upper half is swept, the slot is released and the lower half is swept (recursive
    bisection, a revolve-style schedule)."""

    def __init__(self, dev_adj: "DeviceAdjoint", cap: int, shape, device):
        if cap < 2:
            raise ValueError("max_states must be at least 2")
        self.dev, self.cap = dev_adj, cap
        self.pool = torch.empty((cap,) + tuple(shape), dtype=torch.float64, device=device)
        self.free = list(range(cap - 1, -1, -1))
        self.recomputed = 0

    def take(self) -> int:
        return self.free.pop()

    def give(self, k: int):
        self.free.append(k)

    def advance(self, src: int, n: int, dst: int):
        """Slot dst <- the state n primal iterations after the one in slot src."""
        s = self.dev.solver
        self.dev._enter()
        s.state_from_device(self.pool[src].data_ptr())
        if n:
            s.enqueue(n)
        s.state_to_device(self.pool[dst].data_ptr())
        self.dev._leave()
        self.recomputed += n

    def sweep(self, lo: int, hi: int, slot: int, lam: torch.Tensor, sens: bool):
        n = hi - lo
        if n <= 0:
            return
        if n - 1 <= len(self.free):
            slots = [slot]
            for _ in range(n - 1):
                k = self.take()
                self.advance(slots[-1], 1, k)
                slots.append(k)
            for m in range(n - 1, -1, -1):
                self.dev.step(self.pool[slots[m]], lam, sens)
            for k in slots[1:]:
                self.give(k)
            return
        if len(self.free) == 1:
            # one slot left: each state of the segment recomputed from the snapshot
            k = self.take()
            for m in range(hi - 1, lo, -1):
                self.advance(slot, m - lo, k)
                self.dev.step(self.pool[k], lam, sens)
            self.give(k)
            self.dev.step(self.pool[slot], lam, sens)
            return
        mid = lo + n // 2
        k = self.take()
        self.advance(slot, mid - lo, k)
        self.sweep(mid, hi, k, lam, sens)
        self.give(k)
        self.sweep(lo, mid, slot, lam, sens)


def _transient_gradient_cuda(scheme, objective, p0, t0, amachinit, dy, space, niter, states, lib,
                             max_states=None, record=None) -> dict:
    if scheme.device.type != "cuda":
        raise ValueError("the CUDA adjoint needs a Scheme on a CUDA device")
    params, dy = _leaves(scheme, p0, t0, amachinit, dy)
    space = space or DesignSpace(scheme)
    ni, nj = scheme.ni, scheme.nj
    prm = Params(params[0], params[1], params[2], scheme.flow)
    with torch.no_grad():
        c0 = scheme.cold_state(prm).contiguous()
    dev_adj = DeviceAdjoint(scheme, space, prm, dy, lib)
    if states is None and max_states is not None and max_states < niter + 1:
        try:
            cp = _Checkpoints(dev_adj, max_states, c0.shape, scheme.device)
            root = cp.take()
            cp.pool[root].copy_(c0)
            top = cp.take()
            cp.advance(root, niter, top)  # Q_N (the primal itself)
            QN = cp.pool[top].clone().requires_grad_(True)
            cp.give(top)
            x, y = space.coords(dy)
            J = objective(scheme, QN, scheme.geometry(x, y), prm)
            g = torch.autograd.grad(J, [QN] + params, allow_unused=True)
            grads = [v.detach() if v is not None else torch.zeros_like(p) for v, p in zip(g[1:], params)]
            lam = g[0].detach().contiguous()
            cp.recomputed = 0
            cp.sweep(0, niter, root, lam, True if dy is not None else "scalars")
            sens = dev_adj.sensitivities()
        finally:
            dev_adj.close()
        gp = _parameter_gradient(scheme, space, params, dy, sens, lam)
        grads = [a + b for a, b in zip(grads, gp)]
        out = {"J": float(J.detach()), "dJ_dp0": float(grads[0]), "dJ_dt0": float(grads[1]),
               "dJ_damachinit": float(grads[2]), "lambda0": lam, "states": None,
               "recomputed_iterations": cp.recomputed}
        if dy is not None:
            out["dJ_ddy"] = grads[3].detach().cpu().numpy()
        return out
    recs = None
    try:
        if states is None and record is not False:
            need = niter * dev_adj.solver.adjoint_record_size() * 8
            if record or need < 0.5 * torch.cuda.mem_get_info(scheme.device)[0]:
                st, recs = dev_adj.primal_recorded(c0, niter)
        if recs is not None:
            pass
        elif states is None:
            st = dev_adj.primal(c0, niter)
        elif isinstance(states, torch.Tensor):
            st = states.to(scheme.device, torch.float64).reshape(niter + 1, 5, ni, nj).contiguous()
        else:
            st = torch.tensor(np.asarray(states).reshape(niter + 1, 5, ni, nj), device=scheme.device)
        # dJ/dQ_N and the direct dependence of J on the parameters
        QN = st[niter].clone().requires_grad_(True)
        x, y = space.coords(dy)
        J = objective(scheme, QN, scheme.geometry(x, y), prm)
        g = torch.autograd.grad(J, [QN] + params, allow_unused=True)
        grads = [v.detach() if v is not None else torch.zeros_like(p) for v, p in zip(g[1:], params)]
        lam = g[0].detach().contiguous()
        # without node displacements only the scalar sensitivities are needed
        mode = True if dy is not None else "scalars"
        for n in range(niter - 1, -1, -1):
            dev_adj.step(st[n], lam, mode, rec=recs[n] if recs is not None else None)
        sens = dev_adj.sensitivities()
    finally:
        dev_adj.close()
    gp = _parameter_gradient(scheme, space, params, dy, sens, lam)
    grads = [a + b for a, b in zip(grads, gp)]
    out = {"J": float(J.detach()), "dJ_dp0": float(grads[0]), "dJ_dt0": float(grads[1]),
           "dJ_damachinit": float(grads[2]), "lambda0": lam, "states": st}
    if dy is not None:
        out["dJ_ddy"] = grads[3].detach().cpu().numpy()
    return out


def _fixed_point_cuda(scheme, objective, Qstar, niter, p0, t0, amachinit, dy, space, lib,
                      history_every=1) -> dict:
    if scheme.device.type != "cuda":
        raise ValueError("the CUDA adjoint needs a Scheme on a CUDA device")
    params, dy = _leaves(scheme, p0, t0, amachinit, dy)
    space = space or DesignSpace(scheme)
    prm = Params(params[0], params[1], params[2], scheme.flow)
    Q = Qstar.detach().to(scheme.device, torch.float64).contiguous().requires_grad_(True)
    x, y = space.coords(dy)
    J = objective(scheme, Q, scheme.geometry(x, y), prm)
    gJ = torch.autograd.grad(J, [Q] + params, allow_unused=True)
    djdq = gJ[0].detach().contiguous()
    q = Q.detach()
    dev_adj = DeviceAdjoint(scheme, space, prm, dy, lib)
    hist = []
    try:
        lam = djdq.clone()
        for it in range(niter):
            vj = lam.clone()
            dev_adj.step(q, vj, False, frozen=it > 0)  # Q* is fixed: forward values reused
            new = djdq + vj
            if (it + 1) % history_every == 0 or it == niter - 1:
                hist.append(float(torch.max(torch.abs(new - lam))))
            lam = new
        last = lam.clone()
        dev_adj.step(q, last, True, frozen=niter > 0)  # lambda dG/dp at Q*
        sens = dev_adj.sensitivities()
    finally:
        dev_adj.close()
    gp = _parameter_gradient(scheme, space, params, dy, sens, None)
    grads = []
    for k, p in enumerate(params):
        v = gp[k]
        if gJ[k + 1] is not None:
            v = v + gJ[k + 1]
        grads.append(v)
    out = {"J": float(J.detach()), "dJ_dp0": float(grads[0]), "dJ_dt0": float(grads[1]),
           "dJ_damachinit": float(grads[2]), "residual_history": hist, "lambda": lam}
    if dy is not None:
        out["dJ_ddy"] = grads[3].detach().cpu().numpy()
    return out


class TransientObjective(torch.autograd.Function):
    """J(theta) with theta = [P0, T0, AMACHINIT, dy...]: forward runs the GPU primal
    (FP64, C ABI) from the cold start for ``niter`` iterations and evaluates the
    objective; backward is the checkpointed adjoint sweep of ``transient_gradient``."""

    @staticmethod
    def forward(ctx, theta, scheme, objective, space, niter):
        th = theta.detach().to(torch.float64).cpu()
        dy = th[3:] if th.numel() > 3 else None
        with torch.enable_grad():  # forward of a Function runs with grad mode off
            r = transient_gradient(scheme, objective, float(th[0]), float(th[1]), float(th[2]), dy=dy,
                                   space=space, niter=niter)
        g = [r["dJ_dp0"], r["dJ_dt0"], r["dJ_damachinit"]]
        if dy is not None:
            g += list(r["dJ_ddy"])
        ctx.save_for_backward(torch.tensor(g, dtype=theta.dtype, device=theta.device))
        return torch.tensor(r["J"], dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, gout):
        (g,) = ctx.saved_tensors
        return gout * g, None, None, None, None


# objectives --------------------------------------------------------------------

def wall_force_y(scheme, C, geo, prm, side=1):
    return scheme.wall_force(C, geo, prm, side)[1]


def wall_force_x(scheme, C, geo, prm, side=1):
    return scheme.wall_force(C, geo, prm, side)[0]


def total_pressure_loss(scheme, C, geo, prm):
    return scheme.total_pressure_loss(C, geo, prm)
