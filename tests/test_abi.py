"""The C-ABI library: it loads without a GPU, exports every symbol include/tnsgpu.h
declares, and rejects bad meshes on the host before touching CUDA."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from tnsgpu import _lib, cases
from tnsgpu.solver import make_params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "tnsgpu.h")).read()
    return sorted(set(re.findall(r"\b(tns_[a-z_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = _declared()
    assert len(names) >= 13
    for n in names:
        assert hasattr(L, n), n
    assert set(names) == set(_lib.EXPORTS)


def _create(mesh, flow=None):
    L = _lib.load()
    flow = flow or cases.ramp_flow()
    i32 = lambda a: np.ascontiguousarray(a, np.int32)
    keep = [np.ascontiguousarray(mesh.x), np.ascontiguousarray(mesh.y), i32(mesh.nod.T.reshape(-1)),
            i32(mesh.nc[:, 0]), i32(mesh.nc[:, 1]), i32(mesh.nc[:, 2]), i32(mesh.nc[:, 3]),
            i32(mesh.nparent), i32(mesh.nghost), i32(mesh.ntype), i32(mesh.nside)]
    m = _lib.TnsMesh(mesh.nods, mesh.neles, mesh.nghosts, *(k.ctypes.data for k in keep[:3]),
                     mesh.neles, *(k.ctypes.data for k in keep[3:]))
    p = make_params(flow, 1e-6)
    h = C.c_void_p()
    rc = L.tns_create(C.byref(m), C.byref(p), C.byref(h))
    msg = L.tns_last_error(h).decode() if h else ""
    if h:
        L.tns_destroy(h)
    return rc, msg


@pytest.mark.parametrize("breakage,code", [
    ("type", -2), ("side", -2), ("parent", -2), ("nc", -2), ("collapsed", -2), ("nan_coordinate", -2)])
def test_host_validation_rejects_bad_meshes(breakage, code):
    m = cases.ramp_mesh(6, 4)
    if breakage == "type":
        m.ntype[3] = 1          # no BC type 1 in boundary.f90:33-45
    elif breakage == "side":
        m.nside[0] = 5
    elif breakage == "parent":
        m.nparent[2] = m.nparent[2] + 1
    elif breakage == "nc":
        m.nc[5, 1] = 10_000     # neither a cell nor a ghost
    elif breakage == "collapsed":
        # cell (2, 1): move its nodes N2, N3 onto N1, N4 -> zero area (DT/VOL would divide by 0)
        n = m.nod[2 * 4 + 1] - 1
        m.x = m.x.copy()
        m.y = m.y.copy()
        m.x[n[1]], m.y[n[1]] = m.x[n[0]], m.y[n[0]]
        m.x[n[2]], m.y[n[2]] = m.x[n[3]], m.y[n[3]]
    elif breakage == "nan_coordinate":
        m.y = m.y.copy()
        m.y[7] = float("nan")   # e.g. a corrupted grid.in value
    rc, msg = _create(m)
    assert rc == code, (rc, msg)
    assert msg


def _strip(ni=6):
    """One row of cells: its type-3 ghosts have no cell across the opposite face."""
    xn, yn = np.meshgrid(np.linspace(0.0, 600.0, ni + 1), np.linspace(0.0, 100.0, 2), indexing="ij")
    return cases.multiblock_mesh([(xn, yn)], lambda x, y: 2 if x == 0.0 else 3)


def test_general_meshes_refused_where_the_layout_cannot_follow():
    """A mesh that is not one i x j block takes the general layout; it refuses, before
    any CUDA call, a type-3 ghost with no cell to extrapolate from, and takes mixed
    precision (host checks pass; without a GPU the first CUDA call fails)."""
    rc, msg = _create(_strip())
    assert rc == -3 and "type-3" in msg, (rc, msg)
    f = cases.ramp_flow()
    f_mixed = type(f)(**{**f.__dict__})
    L = _lib.load()
    mesh = cases.backstep_mesh(8, 16, 6, 4)
    i32 = lambda a: np.ascontiguousarray(a, np.int32)
    keep = [np.ascontiguousarray(mesh.x), np.ascontiguousarray(mesh.y), i32(mesh.nod.T.reshape(-1)),
            i32(mesh.nc[:, 0]), i32(mesh.nc[:, 1]), i32(mesh.nc[:, 2]), i32(mesh.nc[:, 3]),
            i32(mesh.nparent), i32(mesh.nghost), i32(mesh.ntype), i32(mesh.nside)]
    m = _lib.TnsMesh(mesh.nods, mesh.neles, mesh.nghosts, *(k.ctypes.data for k in keep[:3]),
                     mesh.neles, *(k.ctypes.data for k in keep[3:]))
    p = make_params(f_mixed, 1e-6, precision=1)
    h = C.c_void_p()
    rc = L.tns_create(C.byref(m), C.byref(p), C.byref(h))
    msg = L.tns_last_error(h).decode()
    L.tns_destroy(h)
    assert rc in (0, -4) and "mixed precision" not in msg, (rc, msg)


def test_general_mesh_passes_host_checks():
    # the backward-facing step: three blocks, not one i x j block
    rc, msg = _create(cases.backstep_mesh(8, 16, 6, 4))
    assert rc in (0, -4), (rc, msg)
    # two interior neighbours swapped: consistent ids, no longer an i x j block
    m = cases.ramp_mesh(6, 4)
    m.nc[9, 1], m.nc[9, 2] = m.nc[9, 2], m.nc[9, 1]
    rc, msg = _create(m)
    assert rc in (0, -4), (rc, msg)


def test_valid_mesh_passes_host_checks():
    rc, msg = _create(cases.ramp_mesh(6, 4))
    # on a machine without a GPU the first CUDA call fails; with one it succeeds
    assert rc in (0, -4), (rc, msg)
