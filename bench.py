#!/usr/bin/env python
"""Benchmark of the RK4 hot path: cell-iterations per second on B200.

Workload (default): the axisymmetric nozzle + plume mesh, 1024 x 384 cells (IAXIS=1,
LOCAL=1, CFL 0.25, cold start at M=0.01), FP64.  One step = one full RK4 iteration
(dissipation pre-pass + 4 stages) over the whole mesh with the state resident in HBM;
L2 is flushed (256 MiB write) between steps outside the timed events.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): every rank solves an independent replica of the mesh (the path has
no exchange step on one GPU: "replicas only"); value = N * cells / max-over-ranks step
time.  --impl reference times the CPU oracle (a line-faithful C restatement of the
reference Fortran, which cannot be compiled here) on the host, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "2d-turbulent-navier-stokes_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "RK4 cell-iters/s on 1 B200, FP32 vs FP64 at equal residual; adjoint/primal time"
UNIT = "cell-iter/s"
# Compulsory DRAM bytes per cell for one launch of each kernel (FP64, 8 B words):
#   dissipation: Q_old 5 + nodes 2 + CFL*DL 1 in, D 5 + DT 1 out                = 14 words
#   viscous    : Q_old 5 + nodes 2 in, VIS 4 out                                = 11 words
#   stage      : Q_in 5 + Q_old 5 + D 5 + VIS 4 + DT 1 + nodes 2 in, Q 5 out    = 27 words
#                (stage 1 reads Q_in = Q_old once: 22 words; mean of the 4 = 25.75)
KERNEL_BYTES_PER_CELL = {"dissipation": 112, "viscous": 88, "stage": 206}
KERNEL_NAMES = {"dissipation": "k_dissipation", "viscous": "k_viscous", "stage": "k_stage"}
# Mixed FP32/FP64 path: D, VIS, DT and the stage increments dQ are FP32 (4 B words):
#   dissipation: Q_old 40 + nodes 16 + CFL*DL 8 in, D 20 + DT 4 out              = 88
#   viscous    : Q_old 40 + nodes 16 in, VIS 16 out                              = 72
#   stage      : Q_old 40 + dQ_in 20 + D 20 + VIS 16 + DT 4 + nodes 16 in,
#                dQ_out 20 out (stage 4: Q_new 40); stage 1 reads no dQ_in        -> mean 143
KERNEL_BYTES_PER_CELL_MX = {"dissipation": 88, "viscous": 72, "stage": 143}
KERNEL_NAMES_MX = {"dissipation": "k_dissipation_mx", "viscous": "k_viscous_mx", "stage": "k_stage_mx"}


def _case(name):
    from tnsgpu import cases, formats
    if name == "nozzle_plume_1024x384":
        m, f = cases.nozzle_plume_mesh(1024, 384), cases.nozzle_plume_flow()
        ri = formats.rinit_cold(f)
        return m, f, formats.cold_state(f, m.neles, ri), ri, \
            "nozzle_plume_1024x384 (IAXIS=1, LOCAL=1, CFL 0.25, cold start M=0.01)"
    if name == "port_4096x1536":
        m, f = cases.port_mesh(4096, 1536), cases.port_flow()
        ri = formats.rinit_cold(f)
        return m, f, formats.cold_state(f, m.neles, ri), ri, \
            "port_4096x1536 (IAXIS=1, type-6 injection, cold start)"
    if name == "ramp_192x64":
        m, f = cases.ramp_mesh(192, 64), cases.ramp_flow()
        c, ri = cases.noisy_restart_state(f, m.neles)
        return m, f, c, ri, "ramp_192x64 (IAXIS=0, seeded restart)"
    raise SystemExit(f"unknown case {name}")


def workload_config(wname, cells, precision, world):
    """The config object both arms print for the same workload."""
    return {"workload": wname, "cells": cells, "precision": precision,
            "step": "one RK4 iteration (dissipation pre-pass + 4 stages)",
            "l2": "flushed between steps (256 MiB write outside the timed events)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(case, kernel):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    try:
        return json.load(open(p)).get(case, {}).get(kernel)
    except Exception:
        return None


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(dev), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            t = [x.strip() for x in line.split(",")]
            if len(t) >= 8:
                rows.append(t)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[4 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def max_over_ranks(x: float, world: int, torch, device) -> float:
    """The largest of every rank's x (a time: the slowest replica sets the pace)."""
    if world <= 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_rate(cells: int, seconds: float, world: int) -> float:
    """Whole-job cell-iterations per second of ``world`` replicas that each advance
    ``cells`` cells by one iteration in ``seconds`` (the max over ranks)."""
    return world * cells / seconds


def time_steps(s, stream, flush, K, W, world, torch):
    """Device time per step (one RK4 iteration; L2 flushed between steps, outside the
    events), max over ranks, plus our launches in the timed region."""
    for _ in range(W):
        flush.zero_()
        s.enqueue(1)
    s.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(K)]
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    l0 = s.launch_count()
    for k in range(K):
        flush.zero_()
        ev[k][0].record(stream)
        s.enqueue(1)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    s.synchronize()
    ms = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / K, world, torch, stream.device)
    return ms, s.launch_count() - l0


def pin_to_gpu_numa_node(dev: int):
    """Restricts this process to the CPUs local to the GPU (NVML), so page-locked host
    buffers live on the GPU's NUMA node and host<->device copies take the short path."""
    try:
        import pynvml
        import torch
        pynvml.nvmlInit()
        # match by UUID: CUDA_VISIBLE_DEVICES renumbers devices, NVML does not
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
        h = pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        words = pynvml.nvmlDeviceGetCpuAffinity(h, (os.cpu_count() + 63) // 64)
        cpus = {w * 64 + b for w, word in enumerate(words) for b in range(64) if word >> b & 1}
        cpus &= os.sched_getaffinity(0)
        if cpus:
            os.sched_setaffinity(0, cpus)
        return sorted(cpus)
    except Exception:
        return None


def run_ours(args, rank, world, dev):
    import numpy as np
    import torch
    from tnsgpu.solver import Solver

    numa_cpus = pin_to_gpu_numa_node(dev)
    mesh, flow, c0, rinit, wname = _case(args.case)
    prec = 1 if args.precision == "mixed" else 0
    kbytes = KERNEL_BYTES_PER_CELL_MX if prec else KERNEL_BYTES_PER_CELL
    knames = KERNEL_NAMES_MX if prec else KERNEL_NAMES
    s = Solver(mesh, flow, rinit, precision=prec)
    # one non-default stream for the solver, the L2 flush and the timing events
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    s.set_stream(stream.cuda_stream)
    s.upload(c0)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    K, W = args.steps, args.warmup
    clocks = Clocks(dev)
    ms, launches = time_steps(s, stream, flush, K, W, world, torch)
    clk = clocks.stop()
    value = replica_rate(mesh.neles, ms * 1e-3, world)

    # per-kernel device times (events around each launch, L2 flushed between iterations)
    s.profile(True)
    P = max(3, min(K, 20))
    for _ in range(P):
        flush.zero_()
        s.enqueue(1)
    s.synchronize()
    kt = s.kernel_times()
    s.profile(False)
    dom = max(("dissipation", "viscous", "stage"), key=lambda k: kt[k][0])
    avg_ms = kt[dom][0] / max(kt[dom][1], 1)
    peak, peak_kind = _peaks()
    bytes_launch = kbytes[dom] * mesh.neles
    achieved = bytes_launch / (avg_ms * 1e-3) / 1e9
    traffic = _traffic(args.case, knames[dom])
    total_kms = sum(kt[k][0] for k in kt) / P
    kernel_split = {k: round(kt[k][0] / P * 1e3, 2) for k in kt if kt[k][1]}

    # end to end through the C ABI: pinned host state -> device, one monitored
    # iteration, the new state and the residual (CDIFF) back to the host
    host = torch.empty((5, mesh.neles), dtype=torch.float64, pin_memory=True)
    host.copy_(torch.from_numpy(np.ascontiguousarray(c0)))
    back = torch.empty((5, mesh.neles), dtype=torch.float64, pin_memory=True)
    ptrs = [host[k].data_ptr() for k in range(5)]
    bptrs = [back[k].data_ptr() for k in range(5)]
    E = max(3, min(K, 200))
    for _ in range(2):
        s.upload_ptrs(ptrs)
        s.run(1, 1)
        s.download_ptrs(bptrs)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(E):
        s.upload_ptrs(ptrs)
        s.run(1, 1)
        s.download_ptrs(bptrs)
    serial_s = max_over_ranks((time.perf_counter() - t0) / E, world, torch, dev)

    # the same steps pipelined over DEPTH handles of the case, each on its own stream:
    # a step's upload, monitored iteration and download are queued at once
    # (tns_upload_state_async, tns_enqueue_monitored, tns_download_state_async) and
    # waited for (tns_synchronize: status word and CDIFF record) only when its handle
    # comes round again, so one step's download overlaps the next steps' uploads and
    # iterations on the two copy engines and the SMs
    DEPTH = 3
    hs = [s] + [Solver(mesh, flow, rinit, precision=prec) for _ in range(DEPTH - 1)]
    for h in hs[1:]:
        h.upload(c0)
        h.prepare()
    outs = [torch.empty((5, mesh.neles), dtype=torch.float64, pin_memory=True) for _ in hs]
    cds = [torch.empty(5, dtype=torch.float64, pin_memory=True) for _ in hs]

    def pipelined(n):
        for k in range(n):
            j = k % DEPTH
            if k >= DEPTH:
                hs[j].synchronize()
            hs[j].upload_async(ptrs)
            hs[j].enqueue_monitored(cds[j].data_ptr())
            hs[j].download_async([outs[j][m].data_ptr() for m in range(5)])
        for h in hs:
            h.synchronize()

    pipelined(2 * DEPTH)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pipelined(E)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / E, world, torch, dev)
    e2e = {"value": replica_rate(mesh.neles, e2e_s, world), "unit": UNIT,
           "h2d_bytes_per_step": 5 * mesh.neles * 8,
           "d2h_bytes_per_step": 5 * mesh.neles * 8 + 5 * 8 + 4,
           "ms_per_step": round(e2e_s * 1e3, 4),
           "step": "upload Q from pinned host, one monitored RK4 iteration, download Q, "
                   "CDIFF record and status word",
           "pipeline": f"{DEPTH} handles of the case in flight, each step's transfers and "
                       "iteration queued asynchronously and synchronised when its handle "
                       "comes round again",
           "serial": {"value": replica_rate(mesh.neles, serial_s, world),
                      "ms_per_step": round(serial_s * 1e3, 4),
                      "step": "the same step through the synchronous calls, one at a time"},
           "host_cpus": f"{len(numa_cpus)} GPU-local" if numa_cpus else "unpinned"}
    for h in hs[1:]:
        h.close()
    s.close()

    # the other precision on the same workload and stream, for the FP32-vs-FP64 metric
    other = None
    if not args.single_precision_mode:
        s2 = Solver(mesh, flow, rinit, precision=1 - prec)
        s2.set_stream(stream.cuda_stream)
        s2.upload(c0)
        ms2, _ = time_steps(s2, stream, flush, K, W, world, torch)
        s2.close()
        other = {"precision": "fp64" if prec else "mixed", "value": replica_rate(mesh.neles, ms2 * 1e-3, world),
                 "ms_per_step": round(ms2, 5), "mixed_over_fp64": (ms2 / ms) if prec == 0 else (ms / ms2)}

    # the same workload through the general-mesh (gather) path: cell and node ids
    # shuffled and every cell's faces rotated, FP64
    gen = None
    if not args.no_general and prec == 0:
        from tnsgpu import cases as cs
        gmesh, gperm = cs.renumbered_mesh(mesh, seed=3)
        gq = np.empty_like(c0)
        gq[:, gperm] = c0
        s3 = Solver(gmesh, flow, rinit, precision=0)
        s3.set_stream(stream.cuda_stream)
        s3.upload(gq)
        ms3, l3 = time_steps(s3, stream, flush, min(K, 300), W, world, torch)
        s3.profile(True)
        for _ in range(3):
            flush.zero_()
            s3.enqueue(1)
        s3.synchronize()
        kt3 = s3.kernel_times()
        s3.profile(False)
        s3.close()
        s4 = Solver(gmesh, flow, rinit, precision=1)
        s4.set_stream(stream.cuda_stream)
        s4.upload(gq)
        ms4, _ = time_steps(s4, stream, flush, min(K, 300), W, world, torch)
        s4.close()
        gen = {"workload": wname + ", cell and node ids shuffled, faces rotated (general-mesh path)",
               "value": replica_rate(mesh.neles, ms3 * 1e-3, world), "ms_per_step": round(ms3, 5),
               "steps": min(K, 300), "launches_per_step": l3 / min(K, 300),
               "over_structured": ms3 / ms,
               "kernel_us_per_iteration": {k: round(kt3[k][0] / 3 * 1e3, 2) for k in kt3 if kt3[k][1]},
               "mixed": {"value": replica_rate(mesh.neles, ms4 * 1e-3, world), "ms_per_step": round(ms4, 5),
                         "mixed_over_fp64": ms4 / ms3}}

    adj = None
    if world == 1 and not args.no_adjoint:
        adj = adjoint_timing(torch, dev)
    bat = None
    if world == 1 and not args.no_batch:
        bat = batch_timing()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(mesh, flow, c0, rinit, budget_s=15.0)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": W, "ms_per_step": round(ms, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64" if prec else "f64",
        "data": "synthetic",
        "config": workload_config(wname, mesh.neles, args.precision, world),
        "roofline": {"bound": "hbm", "kernel": knames[dom], "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind,
                     "bytes_per_launch": bytes_launch, "avg_launch_ms": avg_ms,
                     "traffic": traffic,
                     "iteration_bytes_per_cell": 960,
                     "iteration_frac": value / world * 960 / (peak * 1e9)},
        "kernel_us_per_iteration": kernel_split,
        "device_ms_per_iteration_profiled": round(total_kms, 5),
        "e2e": e2e, "gpu_launches": launches, "clocks": clk,
        "other_precision": other,
        "general_mesh": gen,
        "adjoint": adj,
        "batch": bat,
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def adjoint_timing(torch, dev, K=50, W=5):
    """adjoint/primal time on the discrete-adjoint workload (compression ramp 512 x 192,
    IAXIS=0, LOCAL=1, cold start): one primal RK4 iteration (captured graph) against one
    reverse step of the CUDA adjoint -- with the parameter sensitivities and the
    iteration's forward values recorded by the primal (tns_adjoint_record /
    tns_adjoint_step_recorded), as a transient gradient takes it, or recomputed
    (tns_adjoint_step), and frozen at a fixed
    state, as the fixed-point adjoint takes it.  CUDA events on the adjoint's stream,
    K steps each after W warm-up steps; L2 not flushed on either side (the 512 x 192
    working set is L2-resident for both)."""
    from tnsgpu import adjoint, cases
    mesh, flow = cases.ramp_mesh(512, 192), cases.ramp_flow()
    flow.istart = 0
    sch = adjoint.Scheme(mesh, flow, device=f"cuda:{dev}")
    prm = sch.params()
    da = adjoint.DeviceAdjoint(sch, adjoint.DesignSpace(sch), prm, None)
    try:
        st = da.primal(sch.cold_state(prm).contiguous(), K + W)
        S, s = da.stream, da.solver
        ev = lambda: torch.cuda.Event(enable_timing=True)

        def timed(fn):
            torch.cuda.synchronize()
            a, b = ev(), ev()
            a.record(S)
            for n in range(K):
                fn(n)
            b.record(S)
            torch.cuda.synchronize()
            return a.elapsed_time(b) * 1e3 / K

        s.state_from_device(st[0].data_ptr())
        for _ in range(W):
            s.enqueue(1)
        primal_us = timed(lambda n: s.enqueue(1))
        lam = torch.randn_like(st[0])
        for n in range(W):
            s.adjoint_step(st[n].data_ptr(), lam.data_ptr(), True)
        recompute_us = timed(lambda n: s.adjoint_step(st[K - 1 - n].data_ptr(), lam.data_ptr(), True))
        # the sweep as transient_gradient runs it: a primal that records each iteration's
        # forward values (tns_adjoint_record), then reverse steps that read them
        rs = s.adjoint_record_size()
        recs = torch.empty((K, rs), dtype=torch.float64, device=st.device)
        st2 = torch.empty_like(st[:K + 1])
        st2[0].copy_(st[0])
        s.adjoint_record(st2[0].data_ptr(), st2[1].data_ptr(), recs[0].data_ptr())
        record_us = timed(lambda n: s.adjoint_record(st2[n].data_ptr(), st2[n + 1].data_ptr(), recs[n].data_ptr()))
        for n in range(min(W, K)):
            s.adjoint_step(st2[n].data_ptr(), lam.data_ptr(), True, rec_ptr=recs[n].data_ptr())
        launches0 = s.adjoint_launch_count()
        step_us = timed(lambda n: s.adjoint_step(st2[K - 1 - n].data_ptr(), lam.data_ptr(), True,
                                                 rec_ptr=recs[K - 1 - n].data_ptr()))
        per_step = (s.adjoint_launch_count() - launches0) // K
        # the same sweep for flow-parameter gradients only (no geometric sensitivities)
        for n in range(min(W, K)):
            s.adjoint_step(st2[n].data_ptr(), lam.data_ptr(), "scalars", rec_ptr=recs[n].data_ptr())
        scalars_us = timed(lambda n: s.adjoint_step(st2[K - 1 - n].data_ptr(), lam.data_ptr(), "scalars",
                                                    rec_ptr=recs[K - 1 - n].data_ptr()))
        q = st[K].contiguous()
        s.adjoint_step(q.data_ptr(), lam.data_ptr(), False)
        for _ in range(W):
            s.adjoint_step(q.data_ptr(), lam.data_ptr(), False, True)
        frozen_us = timed(lambda n: s.adjoint_step(q.data_ptr(), lam.data_ptr(), False, True))
        da.sensitivities()
    finally:
        da.close()
    return {"workload": "ramp_512x192 (IAXIS=0, LOCAL=1, cold start)", "steps": K,
            "primal_iteration_us": round(primal_us, 2),
            "primal_record_iteration_us": round(record_us, 2),
            "transient_step_us": round(step_us, 2),
            "transient_step_recompute_us": round(recompute_us, 2),
            "fixed_point_step_us": round(frozen_us, 2),
            "transient_step_over_primal": round(step_us / primal_us, 3),
            "transient_step_flow_parameters_us": round(scalars_us, 2),
            "fixed_point_step_over_primal": round(frozen_us / primal_us, 3),
            "transient_gradient_over_primal": round((record_us + step_us) / primal_us, 3),
            "kernels_per_transient_step": int(per_step)}


def batch_timing(niter=200, monitor=100, stop_ratio=1.0e-5, warmup=16, ncases=64):
    """The batched-sweep workload: ``ncases`` ramp cases from cases.ramp_sweep(seed=0)
    (96x32 .. 512x192 cells, ramp angle, P0, T0 drawn per case), mixed FP32/FP64, cold
    start, convergence masking at ``stop_ratio``.  Each arm first runs ``warmup``
    untimed iterations and captures every CUDA graph it will launch (Solver.prepare,
    Batch.prepare), so no capture falls inside a timed region, then ``niter`` iterations
    with a residual record every ``monitor``: the cases one after another through
    tns_run (the stop criterion checked at every record), and the same cases as one
    batch under schedule 2 (per-case graph branches) and schedule 3 (one persistent
    cooperative launch per run of unmonitored iterations) at the default tile height, and
    under the tile height and schedule tnsgpu.autotune picks by timing a few iterations
    of the sweep (its tuning time reported apart).  Wall time with the device
    synchronised."""
    import numpy as np
    from tnsgpu import cases, formats
    from tnsgpu.batch import Batch
    from tnsgpu.solver import Solver
    sw = cases.ramp_sweep(ncases, seed=0)
    cells = np.array([c.nx * c.ny for c in sw], dtype=np.float64)

    def members(solo_warmup, lib=None):
        out = []
        for c in sw:
            mesh, flow = c.mesh(), c.flow()
            ri = formats.rinit_cold(flow)
            s = Solver(mesh, flow, ri, precision=1, lib=lib)
            s.upload(formats.cold_state(flow, mesh.neles, ri))
            if solo_warmup:
                s.run(warmup, 0)
                s.prepare()
            out.append(s)
        return out

    seq = members(True)
    t0 = time.perf_counter()
    it_seq = []
    for s in seq:
        ref = s.run(1, 1)[0]
        it = 1
        while it < niter:
            n = min(monitor - it % monitor, niter - it)
            rec = s.run(n, n)
            it += n
            if it % monitor == 0 and np.max(rec[-1] / ref) <= stop_ratio:
                break
        it_seq.append(it)
    t_seq = time.perf_counter() - t0
    q_seq = [s.download() for s in seq]
    for s in seq:
        s.close()
    out = {"workload": f"{ncases} ramp cases of cases.ramp_sweep(seed=0), 96x32..512x192, mixed FP32/FP64, "
                       f"cold start + {warmup} untimed iterations",
           "cells_total": int(cells.sum()), "niter": niter, "monitor": monitor, "stop_ratio": stop_ratio,
           "sequential_s": round(t_seq, 4), "sequential_cell_iter_per_s": float(np.sum(cells * it_seq) / t_seq)}
    from tnsgpu import autotune
    t0 = time.perf_counter()
    choice = autotune.tune_batch(lambda lib: members(False, lib), iters=20, warmup=8)
    out["tuned"] = {"ti": choice["ti"], "schedule": choice["schedule"], "tuning_s": round(time.perf_counter() - t0, 2),
                    "trials": [{k: (round(v, 7) if isinstance(v, float) else v) for k, v in t.items()}
                               for t in choice["trials"]]}
    best = None
    arms = [(2, None, "schedule_2"), (3, None, "schedule_3"), (choice["schedule"], choice["lib"], "tuned_run")]
    for sched, lib, key in arms:
        bat = members(False, lib)
        b = Batch(bat, schedule=sched)
        # the warm-up on the batch itself leaves every case where the sequential arm
        # began; prepare() captures this schedule's graphs (monitored and not, the
        # 8-iteration block, both state parities), as the sequential arm's members did
        b.run(warmup, warmup // 2)
        b.prepare()
        l0 = b.launch_count()
        t0 = time.perf_counter()
        r = b.run(niter, monitor, stop_ratio)
        dt = time.perf_counter() - t0
        launches = b.launch_count() - l0
        b.close()
        qb = [s.download() for s in bat]
        same = all(np.array_equal(a, q) for a, q in zip(qb, q_seq))
        diff = max(float(np.max(np.max(np.abs(a - q), axis=1) / np.max(np.abs(q), axis=1))) for a, q in zip(qb, q_seq))
        its = [int(v) for v in r.iterations]
        for s in bat:
            s.close()
        out[key] = {"schedule": sched, "s": round(dt, 4), "launches": int(launches),
                    "cell_iter_per_s": float(np.sum(cells * np.array(its)) / dt),
                    "iterations_equal_sequential": its == it_seq,
                    "states_bitwise_equal_sequential": bool(same), "state_rel_diff_max": diff}
        best = dt if best is None else min(best, dt)
    out["speedup_vs_sequential"] = round(t_seq / best, 3)
    return out


def cpu_baseline(mesh, flow, c0, rinit, budget_s=15.0):
    """The oracle (FP64 C restatement of the reference, single thread) on this host."""
    from oracle.pyoracle import Oracle
    o = Oracle(mesh, flow, rinit, native=True)
    o.set_state(c0)
    t0 = time.perf_counter()
    o.iterate(1, 0)
    one = time.perf_counter() - t0
    n = max(1, int(budget_s / max(one, 1e-6)))
    t0 = time.perf_counter()
    o.iterate(n, 0)
    dt = time.perf_counter() - t0
    return {"value": mesh.neles * n / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"{n} RK4 iterations of the same {mesh.neles}-cell mesh and start "
                      f"state, single thread ({dt:.1f} s), gcc -O3 -march=native "
                      f"-ffp-contract=off built on this host"}


def run_reference(args):
    mesh, flow, c0, rinit, wname = _case(args.case)
    from oracle.pyoracle import Oracle
    o = Oracle(mesh, flow, rinit, native=True)
    o.set_state(c0)
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.warmup, 3))):
        o.iterate(1, 0)
    per = (time.perf_counter() - t0) / max(1, min(args.warmup, 3))
    n = min(args.steps, max(1, int(150.0 / max(per, 1e-6))))
    times = []
    for _ in range(n):
        t = time.perf_counter()
        o.iterate(1, 0)
        times.append(time.perf_counter() - t)
    ms = 1e3 * sum(times) / n
    value = mesh.neles / (ms * 1e-3)
    sample = (f"{n} of {args.steps} requested steps, each one full RK4 iteration of the "
              f"{mesh.neles}-cell mesh, single thread (the reference is serial), gcc -O3 "
              f"-march=native -ffp-contract=off built on this host")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": n,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "impl": "reference",
        "config": workload_config(wname, mesh.neles, args.precision, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--case", default="nozzle_plume_1024x384")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint/primal timing")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched 64-case sweep timing")
    ap.add_argument("--no-general", action="store_true",
                    help="skip the timing of the same workload on the general-mesh path")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="print only the adjoint/primal timing (K = --steps, W = --warmup), for profiling")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64",
                    help="arithmetic of the timed path (the other one is timed too, as other_precision)")
    ap.add_argument("--single-precision-mode", action="store_true",
                    help="time only --precision (no other_precision entry)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    try:
        if args.adjoint_only:
            if rank == 0:
                print(json.dumps({"adjoint": adjoint_timing(torch, local, args.steps, args.warmup)}), flush=True)
            return
        run_ours(args, rank, world, local)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
