"""Case file formats of the reference solver, read and written the way its Fortran does.

* ``flow.in``  -- one list-directed line of 17 values (turbnstwod.f90:20-23, README.md:56-85).
* ``grid.in``  -- ``NODS NELES``, NODS lines ``id x[mm] y[mm] ...``, NELES lines
  ``id N1..N4 NC1..NC4`` (geometry.f90:31-44).  Coordinates are scaled by 0.001
  (geometry.f90:35-36) with the same IEEE multiply.
* ``bc.in``    -- ``NGHOSTS`` then ``NPARENT NGHOST NTYPE NSIDE`` lines (geometry.f90:47-52).
* ``restart.in`` -- NELES lines of C1..C5, then RTRED, NPSEUDO, RINIT, NITEROLD
  (turbnstwod.f90:73-85, 186-195).
* batch manifest -- no reference counterpart: one line per case of a parameter sweep,
  ``name nx ny angle_deg p0 t0 amachinit`` after a ``#`` header line.

Values are written with Python's shortest round-trip ``repr`` so a write/read cycle is
exact; the Fortran list-directed reader accepts that form.
"""
from __future__ import annotations

import dataclasses
import math
import os
from typing import Optional

import numpy as np

MM_TO_M = 0.001  # constants.f90:51


@dataclasses.dataclass
class Mesh:
    """Mesh arrays as COMPUTE_GEOMETRY holds them after reading (1-based ids)."""

    x: np.ndarray  # metres, float64 [nods]
    y: np.ndarray
    nod: np.ndarray  # int32 [neles, 4], 1-based node ids
    nc: np.ndarray  # int32 [neles, 4], 1-based cell / ghost ids
    nparent: np.ndarray  # int32 [nghosts]
    nghost: np.ndarray
    ntype: np.ndarray
    nside: np.ndarray
    x_mm: Optional[np.ndarray] = None  # the file's millimetre values, when known
    y_mm: Optional[np.ndarray] = None
    inj_scale: Optional[np.ndarray] = None  # per bc.in line burn-rate multiplier (type 6)
    shape: Optional[tuple] = None  # (NI, NJ) when generated as one structured block

    @property
    def nods(self) -> int:
        return int(self.x.shape[0])

    @property
    def neles(self) -> int:
        return int(self.nod.shape[0])

    @property
    def nghosts(self) -> int:
        return int(self.nparent.shape[0])


@dataclasses.dataclass
class Flow:
    """The 17 values of flow.in plus the BC 6/7 inputs the reference never assigns."""

    fnamegrid: str = "grid.in"
    fnamebc: str = "bc.in"
    gama: float = 1.4
    amol: float = 28.96
    local: int = 1
    niter: int = 1000
    istart: int = 0
    cfl: float = 0.25
    prandtl: float = 0.72
    prandtlt: float = 0.9
    p0: float = 873500.0
    t0: float = 298.0
    pamb: float = -1.0e5
    amachinit: float = 0.01
    rtred: float = 1.0e-5
    npseudo: int = 1
    iaxis: int = 0
    # BC 6 / 7 extras (no flow.in tokens in the reference)
    tflame: float = 0.0
    ancomb: float = 0.0
    acomb: float = 0.0
    rhoprop: float = 0.0
    pinf: float = 0.0
    aminf: float = 0.0
    deltabl: float = 0.0


def read_flow(path: str) -> Flow:
    with open(path) as fh:
        tok = fh.readline().split()
    if len(tok) < 17:
        raise ValueError(f"{path}: expected 17 values, got {len(tok)}")
    f = Flow()
    f.fnamegrid, f.fnamebc = tok[0], tok[1]
    f.gama, f.amol = float(tok[2]), float(tok[3])
    f.local, f.niter, f.istart = int(tok[4]), int(tok[5]), int(tok[6])
    f.cfl, f.prandtl, f.prandtlt = float(tok[7]), float(tok[8]), float(tok[9])
    f.p0, f.t0, f.pamb = float(tok[10]), float(tok[11]), float(tok[12])
    f.amachinit, f.rtred = float(tok[13]), float(tok[14])
    f.npseudo, f.iaxis = int(tok[15]), int(tok[16])
    return f


def write_flow(path: str, f: Flow) -> None:
    vals = [f.fnamegrid, f.fnamebc, f.gama, f.amol, f.local, f.niter, f.istart, f.cfl,
            f.prandtl, f.prandtlt, f.p0, f.t0, f.pamb, f.amachinit, f.rtred, f.npseudo,
            f.iaxis]
    with open(path, "w") as fh:
        fh.write(" ".join(repr(v) if isinstance(v, float) else str(v) for v in vals) + "\n")
        fh.write("FNAMEGRID, FNAMEBC, GAMA, AMOL, LOCAL, NITER, ISTART, CFL, PRANDTL, "
                 "PRANDTLT, P0, T0, PAMB, AMACHINIT, RTRED, NPSEUDO, IAXIS\n")


def read_grid_bc(grid_path: str, bc_path: str) -> Mesh:
    with open(grid_path) as fh:
        head = fh.readline().split()
        nods, neles = int(head[0]), int(head[1])
        x_mm = np.zeros(nods)
        y_mm = np.zeros(nods)
        for _ in range(nods):
            t = fh.readline().split()
            n = int(t[0])
            x_mm[n - 1] = float(t[1])
            y_mm[n - 1] = float(t[2])
        nod = np.zeros((neles, 4), np.int32)
        nc = np.zeros((neles, 4), np.int32)
        for i in range(neles):
            t = fh.readline().split()
            nod[i] = [int(v) for v in t[1:5]]
            nc[i] = [int(v) for v in t[5:9]]
    with open(bc_path) as fh:
        ng = int(fh.readline().split()[0])
        g = np.zeros((ng, 4), np.int32)
        for i in range(ng):
            g[i] = [int(v) for v in fh.readline().split()[:4]]
    return Mesh(x=x_mm * MM_TO_M, y=y_mm * MM_TO_M, nod=nod, nc=nc, nparent=g[:, 0].copy(),
                nghost=g[:, 1].copy(), ntype=g[:, 2].copy(), nside=g[:, 3].copy(),
                x_mm=x_mm, y_mm=y_mm)


def write_grid_bc(grid_path: str, bc_path: str, m: Mesh) -> None:
    x_mm = m.x_mm if m.x_mm is not None else m.x / MM_TO_M
    y_mm = m.y_mm if m.y_mm is not None else m.y / MM_TO_M
    with open(grid_path, "w") as fh:
        fh.write(f"{m.nods} {m.neles}\n")
        for i in range(m.nods):
            fh.write(f"{i + 1} {float(x_mm[i])!r} {float(y_mm[i])!r} 0.0\n")
        for i in range(m.neles):
            fh.write(" ".join(str(int(v)) for v in (i + 1, *m.nod[i], *m.nc[i])) + "\n")
    with open(bc_path, "w") as fh:
        fh.write(f"{m.nghosts}\n")
        for i in range(m.nghosts):
            fh.write(f"{m.nparent[i]} {m.nghost[i]} {m.ntype[i]} {m.nside[i]}\n")


def read_restart(path: str, neles: int):
    """Returns (C [5, neles] float64, RTRED, NPSEUDO, RINIT, NITEROLD)."""
    with open(path) as fh:
        c = np.zeros((5, neles))
        for i in range(neles):
            t = fh.readline().split()
            c[:, i] = [float(v) for v in t[:5]]
        rtred = float(fh.readline().split()[0])
        npseudo = int(fh.readline().split()[0])
        rinit = float(fh.readline().split()[0])
        niterold = int(fh.readline().split()[0])
    return c, rtred, npseudo, rinit, niterold


def write_restart(path: str, c: np.ndarray, rtred: float, npseudo: int, rinit: float,
                  niterold: int) -> None:
    with open(path, "w") as fh:
        for i in range(c.shape[1]):
            fh.write(" ".join(repr(float(v)) for v in c[:, i]) + "\n")
        fh.write(f"{float(rtred)!r}\n{int(npseudo)}\n{float(rinit)!r}\n{int(niterold)}\n")


def rinit_cold(f: Flow) -> float:
    """RINIT of the isentropic cold start (turbnstwod.f90:53-66)."""
    rr = 8314.0 / f.amol
    dyn = 1.0 + (f.gama - 1.0) * 0.5 * math.pow(f.amachinit, 2.0)
    tinit = f.t0 / dyn
    pinit = f.p0 / math.pow(dyn, f.gama / (f.gama - 1.0))
    rhoinit = pinit / (rr * tinit)
    amu = 0.00000011848 * math.sqrt(f.amol) * math.pow(tinit, 0.6)
    return amu / rhoinit


def cold_state(f: Flow, neles: int, rinit: Optional[float] = None) -> np.ndarray:
    """Uniform isentropic state at AMACHINIT (turbnstwod.f90:53-71), [5, neles]."""
    rr = 8314.0 / f.amol
    cv = rr / (f.gama - 1.0)
    dyn = 1.0 + (f.gama - 1.0) * 0.5 * math.pow(f.amachinit, 2.0)
    tinit = f.t0 / dyn
    pinit = f.p0 / math.pow(dyn, f.gama / (f.gama - 1.0))
    uinit = f.amachinit * math.sqrt(f.gama * rr * tinit)
    vinit = 0.0
    einit = cv * tinit + 0.5 * (math.pow(uinit, 2.0) + math.pow(vinit, 2.0))
    rhoinit = pinit / (rr * tinit)
    if rinit is None:
        rinit = rinit_cold(f)
    c = np.empty((5, neles))
    c[0] = rhoinit
    c[1] = rhoinit * uinit
    c[2] = rhoinit * vinit
    c[3] = rhoinit * einit
    c[4] = rhoinit * rinit
    return c


def write_case(dirpath: str, m: Mesh, f: Flow) -> None:
    os.makedirs(dirpath, exist_ok=True)
    write_grid_bc(os.path.join(dirpath, f.fnamegrid), os.path.join(dirpath, f.fnamebc), m)
    write_flow(os.path.join(dirpath, "flow.in"), f)


MANIFEST_FIELDS = ("name", "nx", "ny", "angle_deg", "p0", "t0", "amachinit")


def write_manifest(path: str, sweep) -> None:
    """Batch manifest of a sweep (objects with the MANIFEST_FIELDS attributes)."""
    with open(path, "w") as fh:
        fh.write("# " + " ".join(MANIFEST_FIELDS) + "\n")
        for c in sweep:
            fh.write(" ".join(repr(getattr(c, k)) if k != "name" else c.name for k in MANIFEST_FIELDS) + "\n")


def read_manifest(path: str) -> list:
    """Rows of a batch manifest as dicts of MANIFEST_FIELDS (ints for nx, ny)."""
    rows = []
    with open(path) as fh:
        for line in fh:
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            t = line.split()
            if len(t) != len(MANIFEST_FIELDS):
                raise ValueError(f"{path}: manifest line needs {len(MANIFEST_FIELDS)} values: {line!r}")
            row = {"name": t[0], "nx": int(t[1]), "ny": int(t[2])}
            for k, v in zip(MANIFEST_FIELDS[3:], t[3:]):
                row[k] = float(v)
            rows.append(row)
    return rows
