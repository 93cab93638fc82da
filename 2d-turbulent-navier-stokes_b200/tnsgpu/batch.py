"""Several cases advanced together on one GPU (tns_batch_* of include/tnsgpu.h).

The reference solves one case per run; a parameter sweep there is a sequence of runs.
``Batch`` co-schedules any number of ``Solver`` handles (different meshes and flow
parameters, one precision mode): every kernel phase of an RK4 iteration is one launch
over the tiles of all active cases.  States move through the member solvers
(``Solver.upload`` / ``download`` / ``primitives``) before and after ``run``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from .solver import Solver


@dataclass
class BatchResult:
    iterations: np.ndarray      # [ncases] iterations each case ran in the call
    records: List[np.ndarray]   # per case [n_records, 5] CDIFF records
    status: np.ndarray          # [ncases] TNS_OK or TNS_ERR_NONFINITE
    reference: np.ndarray       # [ncases, 5] CDIFF reference of the stop criterion
    active: np.ndarray          # [ncases] mask after the call


class Batch:
    def __init__(self, solvers: Sequence[Solver], schedule: int = 0):
        self.solvers = list(solvers)  # keeps the member handles alive
        if not self.solvers:
            raise ValueError("a batch needs at least one case")
        self.L = self.solvers[0].L
        if any(s.L is not self.L for s in self.solvers):
            raise ValueError("batch members must come from one library build")
        arr = (C.c_void_p * len(self.solvers))(*[s.h.value for s in self.solvers])
        self._arr = arr
        b = C.c_void_p()
        rc = self.L.tns_batch_create(arr, len(self.solvers), C.byref(b))
        self.b = b
        self._check(rc)
        self.reference = np.zeros((len(self.solvers), 5))
        if schedule:
            try:
                self.schedule = schedule
            except _lib.TnsError:
                self.close()
                raise

    def _check(self, rc: int):
        if rc != _lib.TNS_OK:
            msg = self.L.tns_batch_last_error(self.b).decode() if self.b else ""
            raise _lib.TnsError(rc, msg)

    @property
    def ncases(self) -> int:
        return len(self.solvers)

    def run(self, niter: int, monitor_every: int = 1000, stop_ratio: float = 0.0,
            raise_on_failure: bool = True) -> BatchResult:
        """Up to niter iterations of every active case.  stop_ratio > 0 masks a case off
        at the first record where max_k CDIFF_k / REF_k <= stop_ratio (REF = the CDIFF
        of its first monitored iteration, kept across calls in ``self.reference``)."""
        n = self.ncases
        maxrec = max(1, niter // monitor_every + 1) if monitor_every > 0 else 1
        out = np.zeros((n, maxrec, 5))
        nrec = np.zeros(n, np.int32)
        iters = np.zeros(n, np.int32)
        status = np.zeros(n, np.int32)
        ref = np.ascontiguousarray(self.reference)
        rc = self.L.tns_batch_run(self.b, int(niter), int(monitor_every), float(stop_ratio),
                                  ref.ctypes.data, out.ctypes.data, maxrec, nrec.ctypes.data,
                                  iters.ctypes.data, status.ctypes.data)
        self.reference = ref
        if rc != _lib.TNS_ERR_NONFINITE or raise_on_failure:
            self._check(rc)
        return BatchResult(iters, [out[k, : nrec[k]] for k in range(n)], status, ref.copy(),
                           self.active())

    @property
    def schedule(self) -> int:
        """0: one launch per phase over all cases' tiles; 1: per-case launches on
        parallel graph branches; 2: as 1 with 8 iterations per graph."""
        return int(self.L.tns_batch_get_schedule(self.b))

    @schedule.setter
    def schedule(self, value: int):
        self._check(self.L.tns_batch_set_schedule(self.b, int(value)))

    def prepare(self):
        """Capture every CUDA graph run() launches under the current schedule and active
        mask now, without running anything (tns_batch_prepare); a change of schedule or
        mask drops them."""
        self._check(self.L.tns_batch_prepare(self.b))

    def set_active(self, mask: Sequence[int]):
        m = np.ascontiguousarray(np.asarray(mask, np.int32))
        if m.shape != (self.ncases,):
            raise ValueError(f"mask needs {self.ncases} entries")
        self._check(self.L.tns_batch_set_active(self.b, m.ctypes.data))

    def active(self) -> np.ndarray:
        m = np.zeros(self.ncases, np.int32)
        self._check(self.L.tns_batch_get_active(self.b, m.ctypes.data))
        return m

    def launch_count(self) -> int:
        return int(self.L.tns_batch_launch_count(self.b))

    def close(self):
        if getattr(self, "b", None) and self.b.value:
            self.L.tns_batch_destroy(self.b)
            self.b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
