"""Quadrilateral meshes and flow cases for the solver.

Every mesh but ``multiblock_mesh``'s is one i x j block numbered the way the reference's grid generators number
theirs (utils/gridgen/ramp.f90:53-63, examples/case1/grid.in): node (i, j) has id
``i*(NJ+1) + j + 1``, cell (i, j) has id ``i*NJ + j + 1`` (j fastest), and cell (i, j)
has nodes N1=(i,j), N2=(i+1,j), N3=(i+1,j+1), N4=(i,j+1) -- faces 1..4 are the j-,
i+, j+ and i- faces.  Ghost cells are numbered NELES+1.. in cell order, sides ascending
within a cell, and listed in bc.in in that order (the order examples/case1/bc.in uses).

Coordinates are generated in millimetres (the grid.in unit) and scaled to metres with
the reference's ``*0.001`` so in-memory meshes equal what the Fortran reads back.

Cases (sizes as named in the solver's benchmark configurations):
  ramp        -- 2-D compression ramp, 1.0 m x 0.3 m, ramp angle from x=0.5 m.
  nozzle_plume-- axisymmetric duct r(x)=0.05+0.03(1-cos(2 pi x/0.4)) over 0..0.4 m
                 (type-5 wall), then the plume region to x=1.0 m, 0.3 m high, all one
                 i x j block: the block's upper boundary leaves the duct lip (0.4, 0.05)
                 on a cosine flare reaching 0.3 m at x=0.5 and is farfield (type 3)
                 from the lip on.  (A steep lip wall inside one block gives cells that
                 make the explicit scheme diverge, on the oracle as well.)
  port        -- axisymmetric 2.0 m x 0.1 m channel with a type-6 injecting port wall.
  nozzle_2d   -- small 2-D converging-diverging channel with the BC layout of the
                 reference's example case (axis 4 / wall 5 / inlet 2 / outflow 3).
  ramp_sweep  -- a seeded parameter sweep of ramp cases (mesh size, ramp angle, P0,
                 T0) for the batched solver.
  backstep    -- a general (multi-block) mesh: a 2-D backward-facing step of three
                 blocks, one of them numbered from another corner (``multiblock_mesh``).
  renumbered  -- any mesh with its cell and node ids shuffled and each cell's faces
                 starting at another corner: the same cells in GAMBIT-like numbering,
                 which the solver runs on its general-mesh path (``renumbered_mesh``).
"""
from __future__ import annotations

import dataclasses
import math
from typing import Callable, Optional

import numpy as np

from .formats import MM_TO_M, Flow, Mesh, cold_state, rinit_cold


def structured_mesh(xn_mm: np.ndarray, yn_mm: np.ndarray,
                    side_type: Callable[[int, np.ndarray], np.ndarray]) -> Mesh:
    """Build grid.in/bc.in arrays for an (NI+1) x (NJ+1) node block.

    ``side_type(side, idx)`` returns the BC type of the ghosts on ``side`` (1..4) for
    the cell indices ``idx`` along that side (i for sides 1/3, j for sides 2/4).
    """
    ni, nj = xn_mm.shape[0] - 1, xn_mm.shape[1] - 1
    if ni < 2 or nj < 2:
        raise ValueError("need at least 2 x 2 cells")
    neles = ni * nj
    ii, jj = np.meshgrid(np.arange(ni), np.arange(nj), indexing="ij")
    ii = ii.ravel()
    jj = jj.ravel()

    def node(i, j):
        return (i * (nj + 1) + j + 1).astype(np.int32)

    def cell(i, j):
        return (i * nj + j + 1).astype(np.int32)

    nod = np.stack([node(ii, jj), node(ii + 1, jj), node(ii + 1, jj + 1), node(ii, jj + 1)],
                   axis=1).astype(np.int32)
    nc = np.stack([cell(ii, jj - 1), cell(ii + 1, jj), cell(ii, jj + 1), cell(ii - 1, jj)],
                  axis=1).astype(np.int32)
    bnd = np.stack([jj == 0, ii == ni - 1, jj == nj - 1, ii == 0], axis=1)
    cid, side = np.nonzero(bnd)  # row-major: cell order, sides ascending
    nghosts = cid.shape[0]
    gid = (neles + 1 + np.arange(nghosts)).astype(np.int32)
    nc[cid, side] = gid
    ntype = np.zeros(nghosts, np.int32)
    for s in range(4):
        sel = side == s
        along = ii[cid[sel]] if s in (0, 2) else jj[cid[sel]]
        ntype[sel] = np.asarray(side_type(s + 1, along), np.int32)
    xm = np.ascontiguousarray(xn_mm.ravel())
    ym = np.ascontiguousarray(yn_mm.ravel())
    return Mesh(x=xm * MM_TO_M, y=ym * MM_TO_M, nod=nod, nc=nc,
                nparent=(cid + 1).astype(np.int32), nghost=gid, ntype=ntype,
                nside=(side + 1).astype(np.int32), x_mm=xm, y_mm=ym, shape=(ni, nj))


def stretch_one_sided(nj: int, beta: float) -> np.ndarray:
    """eta in [0,1] -> tanh clustering toward eta=0."""
    eta = np.linspace(0.0, 1.0, nj + 1)
    return 1.0 - np.tanh(beta * (1.0 - eta)) / math.tanh(beta)


def stretch_two_sided(nj: int, beta: float) -> np.ndarray:
    eta = np.linspace(0.0, 1.0, nj + 1)
    return 0.5 * (1.0 + np.tanh(beta * (eta - 0.5)) / math.tanh(0.5 * beta))


def beta_for_first_cell(nj: int, height: float, first: float) -> float:
    """Solve the one-sided tanh clustering factor giving a first-cell height ``first``."""
    lo, hi = 1e-6, 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        h1 = height * stretch_one_sided(nj, mid)[1]
        if h1 > first:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def ramp_mesh(nx: int, ny: int, angle_deg: float = 10.0, length: float = 1.0,
              height: float = 0.3, x_ramp: float = 0.5, first_cell: float = 1.0e-5,
              wall_dy: Optional[np.ndarray] = None) -> Mesh:
    """Compression ramp: bottom type 5 wall, left type 2, top and right type 3.

    y is tanh-clustered toward the wall with the factor that gives ``first_cell`` metres
    at the inflow station.  ``wall_dy`` (metres, nx+1 values) displaces the wall nodes,
    blended linearly to zero at the top boundary.
    """
    beta = beta_for_first_cell(ny, height, first_cell)
    xs = np.linspace(0.0, length, nx + 1)
    yw = np.where(xs > x_ramp, (xs - x_ramp) * math.tan(math.radians(angle_deg)), 0.0)
    if wall_dy is not None:
        yw = yw + wall_dy
    f = stretch_one_sided(ny, beta)
    xn = np.repeat(xs[:, None], ny + 1, axis=1)
    yn = yw[:, None] + (height - yw[:, None]) * f[None, :]

    def side_type(side, idx):
        return {1: 5, 2: 3, 3: 3, 4: 2}[side] * np.ones_like(idx)

    return structured_mesh(xn * 1000.0, yn * 1000.0, side_type)


def nozzle_plume_mesh(nx: int = 1024, ny: int = 384, flare: float = 0.1,
                      beta: float = 2.5) -> Mesh:
    """Axisymmetric duct + plume as one block (see module docstring).

    Bottom (axis, y=0) type 5; left inlet type 2; top type 5 along the duct (x <= 0.4 m)
    and type 3 beyond the lip; right outflow type 3.
    """
    xs = np.linspace(0.0, 1.0, nx + 1)
    r = 0.05 + 0.03 * (1.0 - np.cos(2.0 * math.pi * np.minimum(xs, 0.4) / 0.4))
    s = np.clip((xs - 0.4) / flare, 0.0, 1.0)
    top = np.where(xs <= 0.4, r, 0.05 + 0.25 * 0.5 * (1.0 - np.cos(math.pi * s)))
    f = stretch_two_sided(ny, beta)
    xn = np.repeat(xs[:, None], ny + 1, axis=1)
    yn = top[:, None] * f[None, :]
    xc = 0.5 * (xs[:-1] + xs[1:])

    def side_type(side, idx):
        if side == 1:
            return 5 * np.ones_like(idx)
        if side == 2:
            return 3 * np.ones_like(idx)
        if side == 4:
            return 2 * np.ones_like(idx)
        return np.where(xc[idx] <= 0.4, 5, 3)

    return structured_mesh(xn * 1000.0, yn * 1000.0, side_type)


def port_mesh(nx: int = 4096, ny: int = 1536, length: float = 2.0, radius: float = 0.1,
              beta: float = 2.0, seed: int = 0, variation: float = 0.02) -> Mesh:
    """Axisymmetric port channel: axis type 5, port wall type 6, head end type 5, exit 3.

    The type-6 ghosts get a burn-rate multiplier 1+U(-variation, variation) drawn from
    ``numpy.random.default_rng(seed)`` in bc.in order.
    """
    xs = np.linspace(0.0, length, nx + 1)
    f = stretch_two_sided(ny, beta)
    xn = np.repeat(xs[:, None], ny + 1, axis=1)
    yn = np.repeat((radius * f)[None, :], nx + 1, axis=0)

    def side_type(side, idx):
        return {1: 5, 2: 3, 3: 6, 4: 5}[side] * np.ones_like(idx)

    m = structured_mesh(xn * 1000.0, yn * 1000.0, side_type)
    rng = np.random.default_rng(seed)
    scale = np.ones(m.nghosts)
    sel = m.ntype == 6
    scale[sel] = 1.0 + rng.uniform(-variation, variation, int(sel.sum()))
    m.inj_scale = scale
    return m


def nozzle_2d_mesh(nx: int = 115, ny: int = 50, beta: float = 2.0) -> Mesh:
    """2-D converging-diverging channel with the example case's BC layout:
    bottom type 4 (symmetry axis), top type 5 wall, left type 2 inlet, right type 3."""
    xs = np.linspace(-0.0678, 0.0578, nx + 1)
    throat = 0.0
    r = np.where(xs < throat, 0.024 + 0.0112 * (1.0 - np.cos(math.pi * xs / xs[0])) * 0.5,
                 0.024 + 0.0006 * (1.0 - np.cos(math.pi * xs / xs[-1])) * 0.5)
    f = np.tanh(beta * np.linspace(0.0, 1.0, ny + 1)) / math.tanh(beta)
    xn = np.repeat(xs[:, None], ny + 1, axis=1)
    yn = r[:, None] * f[None, :]

    def side_type(side, idx):
        return {1: 4, 2: 3, 3: 5, 4: 2}[side] * np.ones_like(idx)

    return structured_mesh(xn * 1000.0, yn * 1000.0, side_type)


# ---------------------------------------------------------------- flow settings

def multiblock_mesh(blocks, bc_type: Callable[[float, float], int], rotate=None) -> Mesh:
    """A general quadrilateral mesh from several structured blocks of nodes.

    ``blocks`` are (xn_mm, yn_mm) node arrays of shape (NI+1, NJ+1), each oriented like
    ``structured_mesh`` (cell (i, j) has nodes (i,j), (i+1,j), (i+1,j+1), (i,j+1), counter-
    clockwise).  Nodes with equal coordinates are one node, so blocks join where their
    node rows coincide.  Cells are numbered block by block (j fastest); ``rotate[b]``
    shifts the local node order of block b's cells cyclically (its faces 1..4 start at
    another corner), as grids converted from other generators number them.  Faces that
    no other cell shares get ghosts, numbered NELES+1.. in cell order, faces ascending,
    with BC type ``bc_type(x_mid_mm, y_mid_mm)`` of the face midpoint.  The result is one
    grid.in / bc.in as the reference reads them (geometry.f90:31-52), not one i x j block.
    """
    node_id: dict = {}
    xs, ys = [], []

    def node(x, y):
        k = (float(x), float(y))
        if k not in node_id:
            node_id[k] = len(xs) + 1
            xs.append(float(x))
            ys.append(float(y))
        return node_id[k]

    nod = []
    for b, (xn, yn) in enumerate(blocks):
        ni, nj = xn.shape[0] - 1, xn.shape[1] - 1
        r = 0 if rotate is None else int(rotate[b]) % 4
        for i in range(ni):
            for j in range(nj):
                q = [node(xn[i, j], yn[i, j]), node(xn[i + 1, j], yn[i + 1, j]),
                     node(xn[i + 1, j + 1], yn[i + 1, j + 1]), node(xn[i, j + 1], yn[i, j + 1])]
                nod.append(q[r:] + q[:r])
    nod = np.asarray(nod, np.int32)
    neles = nod.shape[0]
    edge: dict = {}
    for c in range(neles):
        for k in range(4):
            a, b2 = int(nod[c, k]), int(nod[c, (k + 1) % 4])
            edge.setdefault((min(a, b2), max(a, b2)), []).append((c, k))
    nc = np.zeros((neles, 4), np.int32)
    for faces in edge.values():
        if len(faces) > 2:
            raise ValueError("an edge is shared by more than two cells")
        if len(faces) == 2:
            (c1, k1), (c2, k2) = faces
            nc[c1, k1] = c2 + 1
            nc[c2, k2] = c1 + 1
    xm, ym = np.asarray(xs), np.asarray(ys)
    par, gid, typ, side = [], [], [], []
    for c in range(neles):
        for k in range(4):
            if nc[c, k] == 0:
                g = neles + 1 + len(gid)
                nc[c, k] = g
                a, b2 = nod[c, k] - 1, nod[c, (k + 1) % 4] - 1
                par.append(c + 1)
                gid.append(g)
                side.append(k + 1)
                typ.append(int(bc_type(0.5 * (xm[a] + xm[b2]), 0.5 * (ym[a] + ym[b2]))))
    i32 = lambda v: np.asarray(v, np.int32)
    return Mesh(x=xm * MM_TO_M, y=ym * MM_TO_M, nod=nod, nc=nc, nparent=i32(par), nghost=i32(gid),
                ntype=i32(typ), nside=i32(side), x_mm=xm, y_mm=ym, shape=None)


def backstep_mesh(nx_in: int = 32, nx_out: int = 96, ny_up: int = 24, ny_low: int = 12,
                  length_in: float = 0.2, length_out: float = 0.8, height: float = 0.3,
                  step: float = 0.1) -> Mesh:
    """Backward-facing step, 2-D, three blocks: the inlet channel above the step
    (``length_in`` long, y from ``step`` to ``height``), and downstream of it an upper
    and a lower block (y above and below ``step``); the lower block's cells number their
    nodes from another corner.  Inlet (x=0) type 2, outlet type 3, every other face a
    type-5 wall (channel top and bottom, the step face)."""
    L1, L = length_in * 1000.0, (length_in + length_out) * 1000.0
    h, H = step * 1000.0, height * 1000.0
    grid = lambda x0, x1, nx, y0, y1, ny: np.meshgrid(np.linspace(x0, x1, nx + 1), np.linspace(y0, y1, ny + 1),
                                                      indexing="ij")
    blocks = [grid(0.0, L1, nx_in, h, H, ny_up), grid(L1, L, nx_out, h, H, ny_up),
              grid(L1, L, nx_out, 0.0, h, ny_low)]

    def bc(x, y):
        if x == 0.0:
            return 2
        if x == L:
            return 3
        return 5

    return multiblock_mesh(blocks, bc, rotate=[0, 0, 1])


def ramp_flow(niter: int = 2000, p0: float = 873500.0, t0: float = 298.0) -> Flow:
    """flow.in of the 2-D ramp case: ``grid.in bc.in 1.4 28.96 1 N 1 0.25 0.72 0.9
    P0 T0 -1e5 0.01 1e-5 1 0``."""
    return Flow(gama=1.4, amol=28.96, local=1, niter=niter, istart=1, cfl=0.25,
                prandtl=0.72, prandtlt=0.9, p0=p0, t0=t0, pamb=-1.0e5, amachinit=0.01,
                rtred=1.0e-5, npseudo=1, iaxis=0)


def nozzle_plume_flow(niter: int = 20000) -> Flow:
    return Flow(gama=1.4, amol=28.96, local=1, niter=niter, istart=0, cfl=0.25,
                prandtl=0.72, prandtlt=0.9, p0=873500.0, t0=298.0, pamb=-1.0e5,
                amachinit=0.01, rtred=1.0e-5, npseudo=1, iaxis=1)


def port_flow(niter: int = 10000) -> Flow:
    """Port channel: exit at PAMB=1e5 Pa, injection 10 kg/m^2/s at 2500 K.

    RHOPROP=1800 kg/m^3 with ANCOMB=0 and ACOMB=10/1800 m/s gives RHOPROP*RDOT = 10.
    The initial state is the isentropic cold start from P0=1e5 Pa, T0=2500 K."""
    return Flow(gama=1.4, amol=28.96, local=1, niter=niter, istart=0, cfl=0.25,
                prandtl=0.72, prandtlt=0.9, p0=1.0e5, t0=2500.0, pamb=1.0e5,
                amachinit=0.01, rtred=1.0e-5, npseudo=1, iaxis=1, tflame=2500.0,
                ancomb=0.0, acomb=10.0 / 1800.0, rhoprop=1800.0)


def nozzle_2d_flow(niter: int = 1000) -> Flow:
    """The example case's flow.in values (IAXIS=0, LOCAL=1, cold start)."""
    return Flow(gama=1.4, amol=28.96, local=1, niter=niter, istart=0, cfl=0.25,
                prandtl=0.72, prandtlt=0.9, p0=873500.0, t0=298.0, pamb=-1.0e5,
                amachinit=0.01, rtred=1.0e-5, npseudo=1, iaxis=0)


def noisy_restart_state(f: Flow, neles: int, seed: int = 0, amp: float = 1.0e-3):
    """Cold-start state with C1 scaled by 1+U(-amp, amp) (default_rng(seed)); C2..C5
    unchanged.  Returns (C [5, neles], RINIT)."""
    rinit = rinit_cold(f)
    c = cold_state(f, neles, rinit)
    rng = np.random.default_rng(seed)
    c[0] = c[0] * (1.0 + rng.uniform(-amp, amp, neles))
    return c, rinit


@dataclasses.dataclass
class SweepCase:
    """One ramp case of a parameter sweep (a line of a batch manifest)."""

    name: str
    nx: int
    ny: int
    angle_deg: float
    p0: float
    t0: float
    amachinit: float = 0.01

    def mesh(self) -> Mesh:
        return ramp_mesh(self.nx, self.ny, self.angle_deg)

    def flow(self, niter: int = 2000) -> Flow:
        f = ramp_flow(niter, self.p0, self.t0)
        f.istart = 0
        f.amachinit = self.amachinit
        return f


def ramp_sweep(n: int = 64, seed: int = 0, nx_range=(96, 512), ny_range=(32, 192),
               step: int = 32, angle_range=(5.0, 15.0), p0_range=(2.0e5, 1.0e6),
               t0_range=(250.0, 400.0), amachinit: float = 0.01):
    """n ramp cases drawn from ``numpy.random.default_rng(seed)``: per case, in this
    order, nx and ny uniform over the multiples of ``step`` in their ranges (inclusive),
    then the ramp angle, P0 and T0 uniform in their ranges.  Cold start at AMACHINIT."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(rng.integers(nx_range[0] // step, nx_range[1] // step + 1)) * step
        ny = int(rng.integers(ny_range[0] // step, ny_range[1] // step + 1)) * step
        ang = float(rng.uniform(*angle_range))
        p0 = float(rng.uniform(*p0_range))
        t0 = float(rng.uniform(*t0_range))
        out.append(SweepCase(f"ramp{k:03d}_{nx}x{ny}", nx, ny, ang, p0, t0, amachinit))
    return out


CASES = {
    "ramp_192x64": lambda: (ramp_mesh(192, 64), ramp_flow(2000)),
    "nozzle_plume_1024x384": lambda: (nozzle_plume_mesh(1024, 384), nozzle_plume_flow()),
    "ramp_512x192": lambda: (ramp_mesh(512, 192), ramp_flow(5000)),
    "port_4096x1536": lambda: (port_mesh(4096, 1536), port_flow()),
    "nozzle_2d_115x50": lambda: (nozzle_2d_mesh(115, 50), nozzle_2d_flow()),
}


def renumbered_mesh(mesh: Mesh, seed: int = 0, rotate: bool = True):
    """The same cells, nodes and ghosts under random ids (``default_rng(seed)``) and,
    with ``rotate``, each cell's local node order shifted by a random 0..3 (its NC and
    its ghosts' NSIDE follow).  Ghost ids and the bc.in line order are kept.  Returns
    (mesh, cell_perm) where new cell id cell_perm[c] + 1 holds old cell c + 1, so a state
    q of the old numbering is ``q_new[:, cell_perm] = q``."""
    rng = np.random.default_rng(seed)
    ne, nn = mesh.neles, mesh.nods
    cperm = rng.permutation(ne)          # old cell c -> new index cperm[c]
    nperm = rng.permutation(nn)          # old node n -> new index nperm[n]
    rot = rng.integers(0, 4, ne) if rotate else np.zeros(ne, int)
    inv = np.argsort(cperm)              # new index -> old cell
    r = rot[inv]
    cols = (np.arange(4)[None, :] + r[:, None]) % 4
    old_nod = mesh.nod[inv[:, None], cols]
    old_nc = mesh.nc[inv[:, None], cols]
    nod = nperm[old_nod - 1] + 1
    nc = np.where(old_nc <= ne, cperm[np.clip(old_nc, 1, ne) - 1] + 1, old_nc)
    x = np.zeros(nn)
    y = np.zeros(nn)
    x[nperm] = mesh.x
    y[nperm] = mesh.y
    xm = ym = None
    if mesh.x_mm is not None:
        xm = np.zeros(nn)
        ym = np.zeros(nn)
        xm[nperm] = mesh.x_mm
        ym[nperm] = mesh.y_mm
    par = mesh.nparent - 1
    side = ((mesh.nside - 1 - rot[par]) % 4 + 1).astype(np.int32)
    out = dataclasses.replace(mesh, x=x, y=y, x_mm=xm, y_mm=ym, nod=nod.astype(np.int32),
                              nc=nc.astype(np.int32), nparent=(cperm[par] + 1).astype(np.int32),
                              nside=side, shape=None)
    return out, cperm
