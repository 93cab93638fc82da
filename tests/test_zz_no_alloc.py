"""The allocation-free time step (tns_time_step_noalloc) against the handle-based path.

Callers that cannot allocate device memory while they run -- hosts whose device memory
all comes from one preallocated pool, or plugin hosts that forbid allocation on their
time loop -- get the time step of turbnstwod.f90:97-108 from tns_time_step_noalloc,
whose reduction scratch is a fixed array inside the library.  This test drives it
through the C ABI with device buffers it allocates itself (it is only the checker),
twice in a row, and compares DT and DTMIN with what tns_run computed for the same
state (tns_debug_fetch).  The meshes span one reduction block (960 cells), several
(16 384 cells: 16 partial minima, the last block's reduction through the shared array,
the completion counter left at zero for the next call) and many (393 216 cells).  One
call is also captured into a CUDA graph and replayed, the use the entry point exists for.

This file is collected last so a run that stops at the first failure has run every
other test before it.
"""
import ctypes as C
import math

import numpy as np
import pytest

from tnsgpu import _lib, cases
from tnsgpu.solver import Solver, make_params

pytestmark = pytest.mark.gpu
TOL = 1e-13  # the DT tolerance of the parity tests


def _cfldl(mesh, cfl):
    """CFL*DL per cell in cell-id order, DL = shortest edge (geometry.f90:70-74)."""
    x, y = mesh.x, mesh.y
    n = mesh.nod - 1
    edges = []
    for a, b in ((0, 1), (1, 2), (2, 3), (3, 0)):
        dx = x[n[:, a]] - x[n[:, b]]
        dy = y[n[:, a]] - y[n[:, b]]
        edges.append(np.sqrt(dx * dx + dy * dy))
    dl = np.minimum(np.minimum(np.minimum(edges[0], edges[1]), edges[2]), edges[3])
    return cfl * dl


def _noalloc(torch, q_host, cfldl_dev, params, stream):
    L = _lib.load()
    q = torch.from_numpy(np.ascontiguousarray(q_host)).cuda()
    ncell = q_host.shape[1]
    dt = torch.full((ncell,), math.nan, dtype=torch.float64, device="cuda")
    dtmin = torch.full((1,), math.nan, dtype=torch.float64, device="cuda")
    rc = L.tns_time_step_noalloc(q.data_ptr(), cfldl_dev.data_ptr(), ncell, C.byref(params),
                                 dt.data_ptr(), dtmin.data_ptr(), stream)
    assert rc == 0, _lib.ERRORS.get(rc, rc)
    torch.cuda.synchronize()
    return dt.cpu().numpy(), float(dtmin.cpu().numpy()[0])


@pytest.mark.parametrize("shape", [(48, 20), (256, 64), (1024, 384)])
@pytest.mark.parametrize("local", [1, 0])
def test_noalloc_time_step_matches_handle_path_on_two_calls(local, shape):
    import torch
    mesh = cases.ramp_mesh(*shape)
    flow = cases.ramp_flow()
    flow.local = local
    c0, rinit = cases.noisy_restart_state(flow, mesh.neles)
    params = make_params(flow, rinit)
    cfldl = torch.from_numpy(_cfldl(mesh, flow.cfl)).cuda()
    stream = torch.cuda.current_stream().cuda_stream

    s = Solver(mesh, flow, rinit)
    state = c0
    for call in range(2):
        # handle-based path: DT of the state an iteration starts from
        s.upload(state)
        s.run(1, 0)
        ref = s.debug(2)[0]
        dt, dtmin = _noalloc(torch, state, cfldl, params, stream)
        if local:
            assert np.max(np.abs(dt - ref) / ref) <= TOL, call
            assert abs(dtmin - min(1.0e5, ref.min())) <= TOL * dtmin, call
        else:
            assert abs(dtmin - ref[0]) <= TOL * dtmin, call  # LOCAL=0 runs on DTMIN
            assert abs(dtmin - dt.min()) <= TOL * dtmin, call
        state = s.download()  # the next call starts from a different state
    s.close()


@pytest.mark.parametrize("local", [1, 0])
def test_noalloc_time_step_inside_a_captured_graph(local):
    """One call captured into a CUDA graph after a warm-up call; the graph replayed on two
    states written into its static input, each replay against the handle path."""
    import torch
    mesh = cases.ramp_mesh(256, 64)  # 16 reduction blocks
    flow = cases.ramp_flow()
    flow.local = local
    c0, rinit = cases.noisy_restart_state(flow, mesh.neles)
    params = make_params(flow, rinit)
    L = _lib.load()
    ncell = mesh.neles
    cfldl = torch.from_numpy(_cfldl(mesh, flow.cfl)).cuda()
    q = torch.from_numpy(np.ascontiguousarray(c0)).cuda()
    dt = torch.full((ncell,), math.nan, dtype=torch.float64, device="cuda")
    dtmin = torch.full((1,), math.nan, dtype=torch.float64, device="cuda")

    def call():
        rc = L.tns_time_step_noalloc(q.data_ptr(), cfldl.data_ptr(), ncell, C.byref(params),
                                     dt.data_ptr(), dtmin.data_ptr(),
                                     torch.cuda.current_stream().cuda_stream)
        assert rc == 0, _lib.ERRORS.get(rc, rc)

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        call()  # warm-up outside the capture: the scratch address is looked up here
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        call()

    s = Solver(mesh, flow, rinit)
    state = c0
    for replay in range(2):
        s.upload(state)
        s.run(1, 0)
        ref = s.debug(2)[0]
        q.copy_(torch.from_numpy(np.ascontiguousarray(state)))
        dt.fill_(math.nan)
        dtmin.fill_(math.nan)
        g.replay()
        torch.cuda.synchronize()
        d, m = dt.cpu().numpy(), float(dtmin.cpu().numpy()[0])
        if local:
            assert np.max(np.abs(d - ref) / ref) <= TOL, replay
            assert abs(m - min(1.0e5, ref.min())) <= TOL * m, replay
        else:
            assert abs(m - ref[0]) <= TOL * m, replay
            assert abs(m - d.min()) <= TOL * m, replay
        state = s.download()
    s.close()
    del g


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    L = _lib.load()
    params = make_params(cases.ramp_flow(), 1e-6)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = buf.data_ptr()
    rc = L.tns_time_step_noalloc(p, p, _lib.NOALLOC_MAX_CELLS + 1, C.byref(params), p, p, None)
    assert rc == -7  # TNS_ERR_TOO_LARGE, nothing launched
    assert L.tns_time_step_noalloc(None, p, 10, C.byref(params), p, p, None) == -1
