"""ctypes wrapper of the C oracle (tns_oracle.c).  TEST INFRASTRUCTURE ONLY: used by
tests/, __graft_entry__.smoke() and bench.py's CPU baseline / reference arm as the
checker, never by the product path.  PARITY UNPINNED (see tns_oracle.h)."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libtnsoracle.so")
_NATIVE_PATH = os.path.join(_HERE, "_build", "libtnsoracle_native.so")
_libs = {}


class OraParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "gama", "amol", "cfl", "prandtl", "prandtlt", "p0", "t0", "pamb", "rtred", "rinit",
        "tflame", "ancomb", "acomb", "rhoprop", "pinf", "aminf", "deltabl")] + [
        (n, C.c_int) for n in ("local", "npseudo", "iaxis", "pad_")]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def build_native() -> str:
    """The -march=native copy, compiled on this machine (for the CPU timings only)."""
    subprocess.run(["make", "-s", "-B", "-C", _HERE, "native"], check=True)
    return _NATIVE_PATH


def lib(native: bool = False):
    """The oracle library: the portable build, or with ``native`` the -march=native
    copy, rebuilt on first use in this process so it targets the CPU it runs on."""
    if native not in _libs:
        if native:
            build_native()
        elif not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_NATIVE_PATH if native else _LIB_PATH)
        dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
        ip = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
        L.ora_create.restype = C.c_void_p
        L.ora_create.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, ip, ip, ip, ip, ip, ip,
                                 C.POINTER(OraParams), C.c_void_p]
        L.ora_destroy.argtypes = [C.c_void_p]
        L.ora_cold_start.argtypes = [C.c_void_p, C.c_double]
        L.ora_set_state.argtypes = [C.c_void_p, dp]
        L.ora_get_state.argtypes = [C.c_void_p, dp]
        L.ora_iterate.restype = C.c_int
        L.ora_iterate.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int]
        L.ora_fetch.restype = C.c_int
        L.ora_fetch.argtypes = [C.c_void_p, C.c_char_p, dp, C.c_int]
        L.ora_array_len.restype = C.c_int
        L.ora_array_len.argtypes = [C.c_void_p]
        for n in ("ora_step_dt", "ora_dissipation", "ora_primitive", "ora_boundary",
                  "ora_viscous", "ora_source", "ora_residual"):
            getattr(L, n).argtypes = [C.c_void_p]
        L.ora_update.argtypes = [C.c_void_p, C.c_double]
        L.ora_postprocess.argtypes = [C.c_void_p, dp, dp, dp, dp]
        _libs[native] = L
    return _libs[native]


def params_from_flow(f, rinit: float) -> OraParams:
    p = OraParams()
    for n in ("gama", "amol", "cfl", "prandtl", "prandtlt", "p0", "t0", "pamb", "rtred",
              "tflame", "ancomb", "acomb", "rhoprop", "pinf", "aminf", "deltabl"):
        setattr(p, n, float(getattr(f, n)))
    p.rinit = float(rinit)
    p.local, p.npseudo, p.iaxis = int(f.local), int(f.npseudo), int(f.iaxis)
    return p


class Oracle:
    """One oracle solver instance over a Mesh (formats.Mesh) and Flow."""

    def __init__(self, mesh, flow, rinit: float, native: bool = False):
        self._native = native
        L = lib(native)
        self.mesh, self.flow = mesh, flow
        self._p = params_from_flow(flow, rinit)
        self._inj = None
        if mesh.inj_scale is not None:
            self._inj = np.ascontiguousarray(mesh.inj_scale, np.float64)
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        self._keep = [i32(mesh.nod.reshape(-1)), i32(mesh.nc.reshape(-1))]
        self.h = L.ora_create(mesh.nods, mesh.neles, mesh.nghosts,
                              np.ascontiguousarray(mesh.x, np.float64),
                              np.ascontiguousarray(mesh.y, np.float64),
                              self._keep[0], self._keep[1], i32(mesh.nparent),
                              i32(mesh.nghost), i32(mesh.ntype), i32(mesh.nside),
                              C.byref(self._p),
                              self._inj.ctypes.data if self._inj is not None else None)
        self.nn = L.ora_array_len(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib(self._native).ora_destroy(self.h)
            self.h = None

    def set_state(self, c: np.ndarray):
        lib(self._native).ora_set_state(self.h, np.ascontiguousarray(c, np.float64).reshape(-1))

    def cold_start(self):
        lib(self._native).ora_cold_start(self.h, float(self.flow.amachinit))

    def state(self) -> np.ndarray:
        out = np.zeros(5 * self.mesh.neles)
        lib(self._native).ora_get_state(self.h, out)
        return out.reshape(5, self.mesh.neles)

    def iterate(self, niter: int, monitor_every: int = 1000):
        maxrec = max(1, niter // max(monitor_every, 1) + 1)
        buf = np.zeros(5 * maxrec)
        n = lib(self._native).ora_iterate(self.h, int(niter), int(monitor_every), buf.ctypes.data, maxrec)
        return buf[: 5 * min(n, maxrec)].reshape(-1, 5)

    def fetch(self, name: str) -> np.ndarray:
        out = np.zeros(max(self.nn, self.mesh.nods) + 1)
        n = lib(self._native).ora_fetch(self.h, name.encode(), out, out.shape[0])
        if n < 0:
            raise KeyError(name)
        return out[:n].copy()

    def call(self, routine: str, *args):
        getattr(lib(self._native), "ora_" + routine)(self.h, *args)

    def postprocess(self):
        n = self.mesh.nods
        pn, un, vn, tn = (np.zeros(n) for _ in range(4))
        lib(self._native).ora_postprocess(self.h, pn, un, vn, tn)
        return pn, un, vn, tn
