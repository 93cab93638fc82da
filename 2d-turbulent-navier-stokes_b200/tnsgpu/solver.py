"""Host-side mirror of the reference main program's hot loop over the C ABI.

``Solver`` holds one device handle for a mesh and a flow.in; its calls map one to one
onto the C entry points (include/tnsgpu.h) that replace the RK4 loop of
src/solvers/turbnstwod.f90:95-168 (and the identical turbnsaxis.f90).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .formats import Flow, Mesh


def make_params(flow: Flow, rinit: float, precision: int = 0) -> _lib.TnsParams:
    p = _lib.TnsParams()
    for n in ("gama", "amol", "cfl", "prandtl", "prandtlt", "p0", "t0", "pamb", "rtred",
              "tflame", "ancomb", "acomb", "rhoprop", "pinf", "aminf", "deltabl"):
        setattr(p, n, float(getattr(flow, n)))
    p.rinit = float(rinit)
    p.local, p.npseudo, p.iaxis = int(flow.local), int(flow.npseudo), int(flow.iaxis)
    p.precision = int(precision)
    return p


class Solver:
    """Device solver for one case.  Arrays follow Fortran ids (cell k at index k-1)."""

    def __init__(self, mesh: Mesh, flow: Flow, rinit: float, precision: int = 0,
                 lib: Optional[str] = None):
        """lib: path of the library build to use (a tile-height variant,
        ``_lib.variant_path``); default the TI = 8 build."""
        L = _lib.load(lib)
        self.L, self.mesh, self.flow = L, mesh, flow
        i32 = lambda a: np.ascontiguousarray(a, np.int32)
        # NOD is passed column-major (NOD(I,K) = nod[(K-1)*LD + I-1]) like Fortran holds it
        self._a = dict(x=np.ascontiguousarray(mesh.x, np.float64),
                       y=np.ascontiguousarray(mesh.y, np.float64),
                       nod=i32(mesh.nod.T.reshape(-1)),
                       nc1=i32(mesh.nc[:, 0]), nc2=i32(mesh.nc[:, 1]), nc3=i32(mesh.nc[:, 2]),
                       nc4=i32(mesh.nc[:, 3]), nparent=i32(mesh.nparent),
                       nghost=i32(mesh.nghost), ntype=i32(mesh.ntype), nside=i32(mesh.nside))
        a = self._a
        m = _lib.TnsMesh(mesh.nods, mesh.neles, mesh.nghosts, a["x"].ctypes.data,
                         a["y"].ctypes.data, a["nod"].ctypes.data, mesh.neles,
                         a["nc1"].ctypes.data, a["nc2"].ctypes.data, a["nc3"].ctypes.data,
                         a["nc4"].ctypes.data, a["nparent"].ctypes.data,
                         a["nghost"].ctypes.data, a["ntype"].ctypes.data,
                         a["nside"].ctypes.data)
        self._params = make_params(flow, rinit, precision)
        h = C.c_void_p()
        rc = L.tns_create(C.byref(m), C.byref(self._params), C.byref(h))
        self.h = h
        self._check(rc)
        if mesh.inj_scale is not None:
            self.set_injection_scale(mesh.inj_scale)
        self.maxid = int(max(mesh.neles, int(mesh.nghost.max()) if mesh.nghosts else 0))

    # -- plumbing
    def _check(self, rc: int):
        if rc != _lib.TNS_OK:
            msg = self.L.tns_last_error(self.h).decode() if self.h else ""
            raise _lib.TnsError(rc, msg)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.tns_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- the C entry points
    def set_injection_scale(self, scale: np.ndarray):
        s = np.ascontiguousarray(scale, np.float64)
        self._check(self.L.tns_set_injection_scale(self.h, s.ctypes.data))

    def upload(self, c: np.ndarray):
        """c: [5, NELES] conservative state C1..C5."""
        c = np.ascontiguousarray(c, np.float64)
        self._check(self.L.tns_upload_state(self.h, *(c[k].ctypes.data for k in range(5))))

    def run(self, niter: int, monitor_every: int = 1000) -> np.ndarray:
        maxrec = max(1, niter // monitor_every + 1) if monitor_every > 0 else 1
        buf = np.zeros(5 * maxrec)
        n = C.c_int(0)
        self._check(self.L.tns_run(self.h, int(niter), int(monitor_every), buf.ctypes.data,
                                   maxrec, C.byref(n)))
        return buf[: 5 * n.value].reshape(-1, 5)

    def enqueue(self, niter: int):
        """Asynchronous iterations (no residual monitor); errors surface at synchronize()."""
        self._check(self.L.tns_enqueue(self.h, int(niter)))

    def prepare(self):
        """Capture every CUDA graph run() and enqueue() launch now, without running
        anything, instead of inside the first call that needs each (tns_prepare)."""
        self._check(self.L.tns_prepare(self.h))

    def synchronize(self):
        self._check(self.L.tns_synchronize(self.h))

    def upload_async(self, ptrs):
        """Queue the upload from five page-locked host addresses of NELES doubles and
        return at once (tns_upload_state_async); they must stay valid until
        synchronize()."""
        self._check(self.L.tns_upload_state_async(self.h, *[int(p) for p in ptrs]))

    def enqueue_monitored(self, cdiff_ptr):
        """Queue one monitored iteration whose five CDIFF values arrive at the page-locked
        address ``cdiff_ptr`` by the next synchronize() (tns_enqueue_monitored)."""
        self._check(self.L.tns_enqueue_monitored(self.h, int(cdiff_ptr)))

    def download_async(self, ptrs):
        """Queue the download into five page-locked host addresses of NELES doubles,
        complete at the next synchronize() (tns_download_state_async)."""
        self._check(self.L.tns_download_state_async(self.h, *[int(p) for p in ptrs]))

    def upload_ptrs(self, ptrs):
        """Upload from five host addresses (e.g. page-locked buffers) of NELES doubles."""
        self._check(self.L.tns_upload_state(self.h, *[int(p) for p in ptrs]))

    def download_ptrs(self, ptrs):
        """Download into five host addresses (e.g. page-locked buffers) of NELES doubles."""
        self._check(self.L.tns_download_state(self.h, *[int(p) for p in ptrs]))

    def download(self) -> np.ndarray:
        c = np.zeros((5, self.mesh.neles))
        self._check(self.L.tns_download_state(self.h, *(c[k].ctypes.data for k in range(5))))
        return c

    def primitives(self) -> np.ndarray:
        """[4, maxid] U, V, T, P by Fortran id (cells and ghosts)."""
        out = np.zeros((4, self.maxid))
        self._check(self.L.tns_download_primitives(self.h, *(out[k].ctypes.data for k in range(4))))
        return out

    def node_averages(self) -> np.ndarray:
        """[4, NODS] P, U, V, T node averages of POSTPROCESS (computed on the GPU)."""
        out = np.zeros((4, self.mesh.nods))
        self._check(self.L.tns_node_averages(self.h, *(out[k].ctypes.data for k in range(4))))
        return out

    def boundary_integrals(self, btype: int = 0, side: int = 0) -> np.ndarray:
        """[sum P*SX, sum P*SY, sum RHO*(U*SX+V*SY), sum |S|] over matching boundary faces."""
        out = np.zeros(4)
        self._check(self.L.tns_boundary_integrals(self.h, int(btype), int(side), out.ctypes.data))
        return out

    def total_pressure_sums(self, btype: int = 0, side: int = 0) -> np.ndarray:
        """[sum P0*|MDOT|, sum |MDOT|] over the matching boundary faces (on the GPU)."""
        out = np.zeros(2)
        self._check(self.L.tns_total_pressure_sums(self.h, int(btype), int(side), out.ctypes.data))
        return out

    def total_pressure_loss(self, inlet=(0, 4), outlet=(0, 2)) -> float:
        """1 - (mass-weighted outlet total pressure) / (mass-weighted inlet total pressure),
        the face sets given as (BC type, side), 0 = any."""
        i, o = self.total_pressure_sums(*inlet), self.total_pressure_sums(*outlet)
        return float(1.0 - (o[0] / o[1]) / (i[0] / i[1]))

    def boundary_face_states(self) -> np.ndarray:
        """[5, NGHOSTS] U, V, P, RHO, T of every boundary face in bc.in order (on the GPU)."""
        out = np.zeros((5, self.mesh.nghosts))
        self._check(self.L.tns_boundary_face_states(self.h, out.ctypes.data))
        return out

    def wall_pressure(self, wall_type: int = 5, side: Optional[int] = None) -> np.ndarray:
        """Face pressure of the faces of BC ``wall_type`` (and ``side``), in bc.in order."""
        sel = self.mesh.ntype == wall_type
        if side is not None:
            sel &= self.mesh.nside == side
        return self.boundary_face_states()[2][sel]

    def debug(self, which: int) -> np.ndarray:
        cnt = {0: 5, 1: 4, 2: 1}[which]
        out = np.zeros((cnt, self.mesh.neles))
        self._check(self.L.tns_debug_fetch(self.h, int(which), out.ctypes.data))
        return out

    # -- device-resident state and the discrete adjoint (FP64 handles, (i, j) numbering)
    def state_to_device(self, ptr: int):
        """Copies the state to device memory at ``ptr`` ([5][NELES] doubles), async."""
        self._check(self.L.tns_copy_state_device(self.h, C.c_void_p(int(ptr)), 0))

    def state_from_device(self, ptr: int):
        """Loads the state from device memory at ``ptr`` ([5][NELES] doubles), async."""
        self._check(self.L.tns_copy_state_device(self.h, C.c_void_p(int(ptr)), 1))

    def adjoint_record_size(self) -> int:
        return int(self.L.tns_adjoint_record_size(self.h))

    def adjoint_record(self, q_ptr: int, q_next_ptr: int, rec_ptr: int):
        """One iteration from Q_n (device) to Q_{n+1}, keeping its forward values in the
        record at rec_ptr (tns_adjoint_record)."""
        self._check(self.L.tns_adjoint_record(self.h, C.c_void_p(int(q_ptr)), C.c_void_p(int(q_next_ptr)),
                                              C.c_void_p(int(rec_ptr))))

    def adjoint_step(self, q_ptr: int, lam_ptr: int, sensitivities=False, frozen: bool = False,
                     q_next_ptr: Optional[int] = None, rec_ptr: Optional[int] = None):
        """lambda <- lambda dG/dQ_n for the iteration from Q_n (both device pointers);
        with ``sensitivities`` also accumulates lambda dG/dp (True: all of them;
        "scalars": RTOLERANCE, T0 and S0 only); with ``frozen`` Q_n is the previous
        call's state and its forward values are reused; ``q_next_ptr`` (the next call's
        Q_n) has its forward values computed beside this reverse (tns_adjoint_step_next)."""
        sens = 4 if sensitivities == "scalars" else (1 if sensitivities else 0)
        flags = sens | (2 if frozen else 0)
        if rec_ptr:
            self._check(self.L.tns_adjoint_step_recorded(self.h, C.c_void_p(int(q_ptr)), C.c_void_p(int(rec_ptr)),
                                                         C.c_void_p(int(lam_ptr)), flags))
            return
        nxt = C.c_void_p(int(q_next_ptr)) if q_next_ptr else None
        self._check(self.L.tns_adjoint_step_next(self.h, C.c_void_p(int(q_ptr)) if q_ptr else None, nxt,
                                                 C.c_void_p(int(lam_ptr)), flags))

    def adjoint_sensitivities(self, reset: bool = True) -> np.ndarray:
        n = int(self.L.tns_adjoint_sensitivity_size(self.h))
        out = np.zeros(n)
        self._check(self.L.tns_adjoint_sensitivities(self.h, out.ctypes.data, n, 1 if reset else 0))
        return out

    def adjoint_launch_count(self) -> int:
        return int(self.L.tns_adjoint_launch_count(self.h))

    def set_stream(self, stream_ptr: Optional[int]):
        self._check(self.L.tns_set_stream(self.h, stream_ptr))

    def profile(self, enable: bool):
        self._check(self.L.tns_profile(self.h, 1 if enable else 0))

    def kernel_times(self) -> dict:
        out = {}
        for k, name in enumerate(("dissipation", "viscous", "stage", "dtmin", "gport")):
            ms, n = C.c_double(0), C.c_longlong(0)
            self._check(self.L.tns_kernel_times(self.h, k, C.byref(ms), C.byref(n)))
            out[name] = (ms.value, n.value)
        return out

    def launch_count(self) -> int:
        return int(self.L.tns_launch_count(self.h))
