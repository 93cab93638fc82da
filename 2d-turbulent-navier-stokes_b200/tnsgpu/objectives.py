"""Engineering outputs of a solution: wall pressure, integrated wall force, outlet mass
flow and total-pressure loss.

The reference computes none of these (THRUST is declared, solver_state.f90:40, and
never used).  They are defined here on the solver's own discretisation: a boundary
face carries the average of its parent cell and its ghost (the states the flux
residual uses on that face, residual.f90:33-54), and the face's surface vector S is
geometry.f90:77-99's, so axisymmetric forces and fluxes are per radian.

All functions take a formats.Mesh and the [4, maxid] U, V, T, P array of
Solver.primitives() (cells and ghosts by Fortran id).
"""
from __future__ import annotations

import numpy as np

RUNIV = 8314.0


def face_vectors(mesh, iaxis: int):
    """Surface vector (SX, SY) of every bc.in line's face (outward from the parent)."""
    L = np.arange(mesh.nghosts)
    par = mesh.nparent - 1
    side = mesh.nside - 1
    n1 = mesh.nod[par, side] - 1
    n2 = mesh.nod[par, (side + 1) % 4] - 1
    x1, y1, x2, y2 = mesh.x[n1], mesh.y[n1], mesh.x[n2], mesh.y[n2]
    sx = y2 - y1
    sy = -(x2 - x1)
    if iaxis == 1:
        w = (y1 + y2) * 0.5
        sx, sy = sx * w, sy * w
    return sx[L], sy[L], 0.5 * (x1 + x2), 0.5 * (y1 + y2)


def _face_state(mesh, prims, amol):
    u, v, t, p = prims
    par = mesh.nparent - 1
    gh = mesh.nghost - 1
    rr = RUNIV / amol
    avg = lambda a: 0.5 * (a[par] + a[gh])
    rho = lambda k: p[k] / (rr * t[k])
    return avg(u), avg(v), avg(p), 0.5 * (rho(par) + rho(gh)), avg(t)


def wall_pressure(mesh, prims, amol: float, side: int = None, wall_type: int = 5):
    """Face pressure on every type-5 (wall) face, optionally of one side only.
    Returns (x of the face midpoints, pressure), sorted along x."""
    _, _, pf, _, _ = _face_state(mesh, prims, amol)
    sel = mesh.ntype == wall_type
    if side is not None:
        sel &= mesh.nside == side
    _, _, xm, _ = face_vectors(mesh, 0)
    order = np.argsort(xm[sel])
    return xm[sel][order], pf[sel][order]


def wall_force(mesh, prims, amol: float, iaxis: int, side: int = None, wall_type: int = 5):
    """Pressure force sum(p S) over the wall faces (per radian when IAXIS=1)."""
    _, _, pf, _, _ = _face_state(mesh, prims, amol)
    sx, sy, _, _ = face_vectors(mesh, iaxis)
    sel = np.ones(mesh.nghosts, bool) if wall_type is None else mesh.ntype == wall_type
    if side is not None:
        sel &= mesh.nside == side
    return np.array([np.sum(pf[sel] * sx[sel]), np.sum(pf[sel] * sy[sel])])


def outlet_mass_flow(mesh, prims, amol: float, iaxis: int, side: int = 2):
    """Mass flow sum(rho (u SX + v SY)) out through the faces of one side (outflow)."""
    uf, vf, _, rhof, _ = _face_state(mesh, prims, amol)
    sx, sy, _, _ = face_vectors(mesh, iaxis)
    sel = mesh.nside == side
    return float(np.sum(rhof[sel] * (uf[sel] * sx[sel] + vf[sel] * sy[sel])))


def total_pressure_loss(mesh, prims, amol: float, gama: float, iaxis: int, inlet_side: int = 4,
                        outlet_side: int = 2):
    """1 - (mass-weighted outlet total pressure) / (mass-weighted inlet total pressure)."""
    uf, vf, pf, rhof, tf = _face_state(mesh, prims, amol)
    sx, sy, _, _ = face_vectors(mesh, iaxis)
    rr = RUNIV / amol
    mach2 = (uf * uf + vf * vf) / (gama * rr * tf)
    p0 = pf * (1.0 + 0.5 * (gama - 1.0) * mach2) ** (gama / (gama - 1.0))
    mdot = np.abs(rhof * (uf * sx + vf * sy))

    def mean(side):
        sel = mesh.nside == side
        return np.sum(p0[sel] * mdot[sel]) / np.sum(mdot[sel])

    return float(1.0 - mean(outlet_side) / mean(inlet_side))
