"""ctypes binding of libtnsgpu.so (the C ABI declared in include/tnsgpu.h).

The library is built in-tree (``tnsgpu.build.build_library``); there is no fallback:
if the shared object is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# TNSGPU_LIB names another build of the library to load by default
LIB_PATH = os.environ.get("TNSGPU_LIB") or os.path.join(HERE, "libtnsgpu.so")
# tile-height variants of the same library (TI rows of 32 cells per tile); the default
# build is TI = 8
TILE_VARIANTS = {8: LIB_PATH, 4: os.path.join(HERE, "libtnsgpu_ti4.so"),
                 16: os.path.join(HERE, "libtnsgpu_ti16.so")}


def variant_path(ti: int) -> str:
    if ti not in TILE_VARIANTS:
        raise ValueError(f"no tile variant TI={ti}; built: {sorted(TILE_VARIANTS)}")
    return TILE_VARIANTS[ti]

TNS_OK = 0
ERRORS = {-1: "TNS_ERR_ARG", -2: "TNS_ERR_MESH", -3: "TNS_ERR_UNSUPPORTED",
          -4: "TNS_ERR_CUDA", -5: "TNS_ERR_NONFINITE", -6: "TNS_ERR_STATE",
          -7: "TNS_ERR_TOO_LARGE"}
for _code, _name in ERRORS.items():
    globals()[_name] = _code
NOALLOC_MAX_CELLS = 256 * 4 * 8192

# every symbol include/tnsgpu.h declares
EXPORTS = ("tns_create", "tns_set_injection_scale", "tns_upload_state", "tns_run",
           "tns_enqueue", "tns_prepare", "tns_synchronize", "tns_upload_state_async", "tns_enqueue_monitored",
           "tns_download_state_async", "tns_download_state", "tns_download_primitives", "tns_debug_fetch",
           "tns_set_stream", "tns_profile", "tns_kernel_times", "tns_launch_count",
           "tns_last_error", "tns_destroy", "tns_time_step_noalloc", "tns_node_averages",
           "tns_boundary_integrals", "tns_total_pressure_sums", "tns_boundary_face_states", "tns_batch_create", "tns_batch_run", "tns_batch_set_active",
           "tns_batch_get_active", "tns_batch_set_schedule", "tns_batch_get_schedule", "tns_batch_prepare",
           "tns_batch_launch_count", "tns_debug_math", "tns_batch_last_error", "tns_batch_destroy",
           "tns_adjoint_enable", "tns_adjoint_step", "tns_adjoint_step_next", "tns_adjoint_sensitivity_size",
           "tns_adjoint_record_size", "tns_adjoint_record", "tns_adjoint_step_recorded",
           "tns_adjoint_sensitivities", "tns_adjoint_launch_count", "tns_copy_state_device")
NOT_INT = ("tns_launch_count", "tns_last_error", "tns_destroy", "tns_batch_launch_count",
           "tns_batch_last_error", "tns_batch_destroy", "tns_adjoint_sensitivity_size", "tns_adjoint_record_size",
           "tns_adjoint_launch_count")


class TnsMesh(C.Structure):
    _fields_ = [("nods", C.c_int), ("neles", C.c_int), ("nghosts", C.c_int),
                ("x", C.c_void_p), ("y", C.c_void_p), ("nod", C.c_void_p), ("ld_nod", C.c_int),
                ("nc1", C.c_void_p), ("nc2", C.c_void_p), ("nc3", C.c_void_p),
                ("nc4", C.c_void_p), ("nparent", C.c_void_p), ("nghost", C.c_void_p),
                ("ntype", C.c_void_p), ("nside", C.c_void_p)]


class TnsParams(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "gama", "amol", "cfl", "prandtl", "prandtlt", "p0", "t0", "pamb", "rtred", "rinit",
        "tflame", "ancomb", "acomb", "rhoprop", "pinf", "aminf", "deltabl")] + [
        (n, C.c_int) for n in ("local", "npseudo", "iaxis", "precision")]


class TnsError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


_libs = {}


def load(path: str = None):
    """Load the library (raises OSError when it is missing); one instance per path."""
    path = os.path.abspath(path or LIB_PATH)
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        raise OSError(f"{path} is missing: build it with tnsgpu.build.build_library()")
    L = C.CDLL(path)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_void_p
    L.tns_create.argtypes = [C.POINTER(TnsMesh), C.POINTER(TnsParams), C.POINTER(vp)]
    L.tns_set_injection_scale.argtypes = [vp, dp]
    L.tns_upload_state.argtypes = [vp, dp, dp, dp, dp, dp]
    L.tns_run.argtypes = [vp, ip, ip, dp, ip, C.POINTER(C.c_int)]
    L.tns_enqueue.argtypes = [vp, ip]
    L.tns_prepare.argtypes = [vp]
    L.tns_upload_state_async.argtypes = [vp, vp, vp, vp, vp, vp]
    L.tns_enqueue_monitored.argtypes = [vp, vp]
    L.tns_download_state_async.argtypes = [vp, vp, vp, vp, vp, vp]
    L.tns_synchronize.argtypes = [vp]
    L.tns_download_state.argtypes = [vp, dp, dp, dp, dp, dp]
    L.tns_download_primitives.argtypes = [vp, dp, dp, dp, dp]
    L.tns_debug_fetch.argtypes = [vp, ip, dp]
    L.tns_node_averages.argtypes = [vp, dp, dp, dp, dp]
    L.tns_boundary_integrals.argtypes = [vp, ip, ip, dp]
    L.tns_total_pressure_sums.argtypes = [vp, ip, ip, dp]
    L.tns_boundary_face_states.argtypes = [vp, dp]
    L.tns_set_stream.argtypes = [vp, vp]
    L.tns_profile.argtypes = [vp, ip]
    L.tns_kernel_times.argtypes = [vp, ip, C.POINTER(C.c_double), C.POINTER(C.c_longlong)]
    L.tns_launch_count.argtypes = [vp]
    L.tns_launch_count.restype = C.c_longlong
    L.tns_last_error.argtypes = [vp]
    L.tns_last_error.restype = C.c_char_p
    L.tns_destroy.argtypes = [vp]
    L.tns_destroy.restype = None
    L.tns_time_step_noalloc.argtypes = [vp, vp, C.c_longlong, C.POINTER(TnsParams), vp, vp, vp]
    L.tns_batch_create.argtypes = [vp, ip, C.POINTER(vp)]
    L.tns_batch_run.argtypes = [vp, ip, ip, C.c_double, dp, dp, ip, vp, vp, vp]
    L.tns_batch_set_active.argtypes = [vp, vp]
    L.tns_batch_get_active.argtypes = [vp, vp]
    L.tns_batch_set_schedule.argtypes = [vp, ip]
    L.tns_debug_math.argtypes = [ip, C.c_longlong, dp, dp, dp]
    L.tns_batch_get_schedule.argtypes = [vp]
    L.tns_batch_prepare.argtypes = [vp]
    L.tns_batch_launch_count.argtypes = [vp]
    L.tns_batch_launch_count.restype = C.c_longlong
    L.tns_batch_last_error.argtypes = [vp]
    L.tns_batch_last_error.restype = C.c_char_p
    L.tns_batch_destroy.argtypes = [vp]
    L.tns_batch_destroy.restype = None
    L.tns_adjoint_enable.argtypes = [vp]
    L.tns_adjoint_step.argtypes = [vp, vp, vp, ip]
    L.tns_adjoint_step_next.argtypes = [vp, vp, vp, vp, ip]
    L.tns_adjoint_step_recorded.argtypes = [vp, vp, vp, vp, ip]
    L.tns_adjoint_record.argtypes = [vp, vp, vp, vp]
    L.tns_adjoint_record_size.argtypes = [vp]
    L.tns_adjoint_record_size.restype = C.c_longlong
    L.tns_adjoint_sensitivity_size.argtypes = [vp]
    L.tns_adjoint_sensitivity_size.restype = C.c_longlong
    L.tns_adjoint_sensitivities.argtypes = [vp, vp, C.c_longlong, ip]
    L.tns_adjoint_launch_count.argtypes = [vp]
    L.tns_adjoint_launch_count.restype = C.c_longlong
    L.tns_copy_state_device.argtypes = [vp, vp, ip]
    for n in EXPORTS:
        if n not in NOT_INT:
            getattr(L, n).restype = C.c_int
    _libs[path] = L
    return L


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data
