"""CPU oracle checks.  The reference ships no golden vectors and cannot be compiled here
(no Fortran compiler), so the oracle is pinned by invariants of the discretisation and
by a literal per-routine transcription on a tiny mesh."""
import math

import numpy as np
import pytest

from oracle.pyoracle import Oracle
from tnsgpu import cases, formats


def _quiescent(mesh, flow):
    ri = formats.rinit_cold(flow)
    f = formats.Flow(**{**flow.__dict__, "amachinit": 0.0})
    return formats.cold_state(f, mesh.neles, ri), ri


def test_quiescent_state_is_preserved():
    # fluid at rest inside symmetry/wall boundaries: every flux balances, D = VIS = 0
    m = cases.ramp_mesh(16, 8, angle_deg=0.0)
    m.ntype[:] = np.where(m.nside == 1, 5, 4)
    f = cases.ramp_flow()
    c0, ri = _quiescent(m, f)
    o = Oracle(m, f, ri)
    o.set_state(c0)
    o.iterate(10, 0)
    q = o.state()
    assert np.allclose(q[0], c0[0], rtol=1e-12, atol=0)
    assert np.max(np.abs(q[1:3])) < 1e-9 * np.max(np.abs(c0[3]))


def test_mirror_symmetric_channel():
    # a channel symmetric about its mid-line stays mirror-symmetric
    ni, nj = 12, 10
    xs = np.linspace(0.0, 0.2, ni + 1)
    ys = np.linspace(0.0, 0.05, nj + 1)
    xn, yn = np.meshgrid(xs, ys, indexing="ij")
    m = cases.structured_mesh(xn * 1000, yn * 1000,
                              lambda s, idx: {1: 5, 2: 3, 3: 5, 4: 2}[s] * np.ones_like(idx))
    # node averages at corners depend on bc.in order (viscous.f90:116-121 overrides): list
    # the top-right corner cell's wall ghost before its outflow ghost, mirroring the
    # bottom-right corner's order, so the mirrored problem is the same problem
    last = np.nonzero(m.nparent == m.neles)[0]
    assert m.nside[last].tolist() == [2, 3]
    order = np.arange(m.nghosts)
    order[last] = last[::-1]
    for k in ("nparent", "nghost", "ntype", "nside"):
        setattr(m, k, getattr(m, k)[order].copy())
    f = cases.nozzle_2d_flow()
    ri = formats.rinit_cold(f)
    o = Oracle(m, f, ri)
    o.set_state(formats.cold_state(f, m.neles, ri))
    o.iterate(30, 0)
    q = o.state().reshape(5, ni, nj)
    mir = q[:, :, ::-1]
    scale = np.max(np.abs(q), axis=(1, 2))
    for k in (0, 1, 3, 4):
        assert np.max(np.abs(q[k] - mir[k])) <= 1e-12 * scale[k]
    assert np.max(np.abs(q[2] + mir[2])) <= 1e-12 * scale[1]


def _literal_dt_dissipation(mesh, flow, c, ri):
    """Independent transcription of turbnstwod.f90:97-114 and solver_state.f90:70-225 with
    1-based Python arrays, written from the Fortran without looking at the C oracle."""
    nn = max(mesh.neles, int(mesh.nghost.max()))
    RR = 8314.0 / flow.amol
    CV = RR / (flow.gama - 1.0)
    RTOL = ri * flow.rtred
    C = [np.zeros(nn + 1) for _ in range(5)]
    for k in range(5):
        C[k][1:mesh.neles + 1] = c[k]
    X = np.r_[0.0, mesh.x]
    Y = np.r_[0.0, mesh.y]
    NOD = np.zeros((nn + 1, 4), int)
    NOD[1:mesh.neles + 1] = mesh.nod
    NC = np.zeros((nn + 1, 4), int)
    NC[1:mesh.neles + 1] = mesh.nc
    VOL = np.zeros(nn + 1)
    DL = np.zeros(nn + 1)
    for I in range(1, mesh.neles + 1):
        n1, n2, n3, n4 = NOD[I]
        X1, X2, X3, X4 = X[n1], X[n2], X[n3], X[n4]
        Y1, Y2, Y3, Y4 = Y[n1], Y[n2], Y[n3], Y[n4]
        DL[I] = min(math.sqrt((X1 - X2) * (X1 - X2) + (Y1 - Y2) * (Y1 - Y2)),
                    math.sqrt((X2 - X3) * (X2 - X3) + (Y2 - Y3) * (Y2 - Y3)),
                    math.sqrt((X3 - X4) * (X3 - X4) + (Y3 - Y4) * (Y3 - Y4)),
                    math.sqrt((X4 - X1) * (X4 - X1) + (Y4 - Y1) * (Y4 - Y1)))
        VOL[I] = abs(0.5 * ((X3 - X1) * (Y4 - Y2) - (X4 - X2) * (Y3 - Y1)))
    for L in range(mesh.nghosts):
        VOL[mesh.nghost[L]] = VOL[mesh.nparent[L]]
    P = np.zeros(nn + 1)
    DT = np.zeros(nn + 1)
    for I in range(1, mesh.neles + 1):
        RHO = C[0][I]
        U = C[1][I] / RHO
        V = C[2][I] / RHO
        VEL = math.sqrt(U * U + V * V)
        E = C[3][I] / RHO
        T = (E - 0.5 * (U * U + V * V)) / CV
        P[I] = RHO * RR * T
        DT[I] = flow.cfl * DL[I] / (abs(VEL) + math.sqrt(flow.gama * RR * T))
    for L in range(mesh.nghosts):
        NG, NP = mesh.nghost[L], mesh.nparent[L]
        P[NG] = P[NP]
        DT[NG] = DT[NP]
        for k in range(5):
            C[k][NG] = C[k][NP]
    ANU = np.zeros(nn + 1)
    ANURT = np.zeros(nn + 1)
    D2Q = [np.zeros(nn + 1) for _ in range(5)]
    for I in range(1, mesh.neles + 1):
        n = NC[I]
        ANU[I] = sum(abs(P[k] - P[I]) for k in n) / sum(abs(P[k] + P[I]) for k in n)
        ANURT[I] = (sum(abs(C[4][k] - C[4][I]) for k in n) /
                    max(sum(abs(C[4][k] + C[4][I]) for k in n), 8.0 * C[0][I] * RTOL))
        for m in range(5):
            D2Q[m][I] = C[m][n[0]] + C[m][n[1]] + C[m][n[2]] + C[m][n[3]] - 4.0 * C[m][I]
    for L in range(mesh.nghosts):
        NG, NP = mesh.nghost[L], mesh.nparent[L]
        ANU[NG] = ANU[NP]
        for m in range(5):
            D2Q[m][NG] = D2Q[m][NP]
    D = np.zeros((5, mesh.neles))
    for I in range(1, mesh.neles + 1):
        for m in range(5):
            S = ANURT if m == 4 else ANU
            d2 = d4 = 0.0
            for k in NC[I]:
                e2 = 0.25 * max(S[I], S[k])
                e4 = max(0.0, 0.00390625 - e2)
                d24 = 0.5 * (VOL[I] / DT[I] + VOL[k] / DT[k])
                d2 += e2 * d24 * (C[m][k] - C[m][I])
                d4 += e4 * d24 * (D2Q[m][k] - D2Q[m][I])
            D[m, I - 1] = d2 - d4
    return DT[1:mesh.neles + 1], D


def test_oracle_matches_literal_dt_and_dissipation():
    m = cases.ramp_mesh(7, 5)
    f = cases.ramp_flow()
    c, ri = cases.noisy_restart_state(f, m.neles, amp=0.05)
    c[1] *= 1.0 + 0.3 * np.random.default_rng(3).uniform(-1, 1, m.neles)
    dt_ref, d_ref = _literal_dt_dissipation(m, f, c, ri)
    o = Oracle(m, f, ri)
    o.set_state(c)
    o.call("step_dt")
    o.call("dissipation")
    assert np.allclose(o.fetch("DT")[:m.neles], dt_ref, rtol=1e-14, atol=0)
    for k in range(5):
        got = o.fetch(f"D24{k + 1}")[:m.neles]
        scale = np.max(np.abs(d_ref[k])) or 1.0
        assert np.max(np.abs(got - d_ref[k])) <= 1e-13 * scale, k


def test_axis_wall_sensitivity_is_a_property_of_the_scheme():
    """With IAXIS=1 and the axis as a type-5 wall, a 1e-15 relative input change moves C5
    by orders of magnitude more after one iteration (the PHI>0 switch of DEE,
    source_terms.f90:71-72, acting on roundoff-level radial velocity); with the axis as
    type 4 it does not.  GPU parity tests for such cases are compared against this envelope."""
    f = cases.port_flow()
    for axis_type, big in ((5, True), (4, False)):
        m = cases.port_mesh(32, 12)
        m.ntype[(m.ntype == 5) & (m.nside == 1)] = axis_type
        ri = formats.rinit_cold(f)
        c0 = formats.cold_state(f, m.neles, ri)
        c1 = c0 * (1 + 1e-15 * np.random.default_rng(1).standard_normal(c0.shape))
        out = []
        for c in (c0, c1):
            o = Oracle(m, f, ri)
            o.set_state(c)
            o.iterate(1, 0)
            out.append(o.state())
        rel = np.max(np.abs(out[0][4] - out[1][4])) / np.max(np.abs(out[0][4]))
        assert (rel > 1e-9) == big, (axis_type, rel)
