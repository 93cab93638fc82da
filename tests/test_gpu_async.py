"""Asynchronous transfers and monitored iterations (tns_upload_state_async,
tns_enqueue_monitored, tns_download_state_async) against the synchronous calls.

A pipelined caller keeps several handles in flight: each step uploads a state from
page-locked host memory, runs one monitored iteration and downloads the new state and
its residual record, and the next step on another handle starts before this one ends.
Every step's state and CDIFF record must equal, bit for bit, what tns_upload_state +
tns_run(h, 1, 1) + tns_download_state give for the same input.
"""
import numpy as np
import pytest

from tnsgpu import _lib, cases
from tnsgpu.solver import Solver

pytestmark = pytest.mark.gpu


def _pinned(torch, shape):
    return torch.empty(shape, dtype=torch.float64, pin_memory=True)


def _sync_step(mesh, flow, ri, precision, q):
    s = Solver(mesh, flow, ri, precision=precision)
    s.upload(q)
    rec = s.run(1, 1)
    out = s.download()
    s.close()
    return out, rec[0]


@pytest.mark.parametrize("precision", [0, 1])
def test_pipelined_steps_equal_synchronous_steps(precision):
    import torch
    mesh = cases.ramp_mesh(96, 40)
    flow = cases.ramp_flow()
    states = []
    for seed in range(5):
        c0, ri = cases.noisy_restart_state(flow, mesh.neles, seed=seed)
        states.append(c0)
    ri = cases.noisy_restart_state(flow, mesh.neles, seed=0)[1]
    depth = 3
    handles = [Solver(mesh, flow, ri, precision=precision) for _ in range(depth)]
    for h in handles:
        h.upload(states[0])  # a state for prepare()
        h.prepare()
    ins = [_pinned(torch, (5, mesh.neles)) for _ in states]
    for t, q in zip(ins, states):
        t.copy_(torch.from_numpy(np.ascontiguousarray(q)))
    outs = [_pinned(torch, (5, mesh.neles)) for _ in states]
    cds = [_pinned(torch, (5,)) for _ in states]
    busy = [None] * depth
    for k in range(len(states)):
        h = handles[k % depth]
        if busy[k % depth] is not None:
            h.synchronize()
        h.upload_async([ins[k][m].data_ptr() for m in range(5)])
        h.enqueue_monitored(cds[k].data_ptr())
        h.download_async([outs[k][m].data_ptr() for m in range(5)])
        busy[k % depth] = k
    for h in handles:
        h.synchronize()
    for k, q in enumerate(states):
        ref_q, ref_rec = _sync_step(mesh, flow, ri, precision, q)
        np.testing.assert_array_equal(outs[k].numpy(), ref_q, err_msg=f"step {k}")
        np.testing.assert_array_equal(cds[k].numpy(), ref_rec, err_msg=f"step {k}")
    for h in handles:
        h.close()


def test_async_calls_refuse_what_they_cannot_do():
    import torch
    mesh = cases.ramp_mesh(48, 20)
    flow = cases.ramp_flow()
    c0, ri = cases.noisy_restart_state(flow, mesh.neles)
    s = Solver(mesh, flow, ri)
    pinned = _pinned(torch, (5, mesh.neles))
    pinned.copy_(torch.from_numpy(np.ascontiguousarray(c0)))
    pageable = np.ascontiguousarray(c0)
    cd = _pinned(torch, (5,))
    # pageable host arrays: TNS_ERR_ARG, nothing queued
    with pytest.raises(_lib.TnsError) as e:
        s.upload_async([pageable[m].ctypes.data for m in range(5)])
    assert e.value.code == _lib.TNS_ERR_ARG
    s.upload_async([pinned[m].data_ptr() for m in range(5)])
    with pytest.raises(_lib.TnsError) as e:
        s.enqueue_monitored(pageable[0].ctypes.data)
    assert e.value.code == _lib.TNS_ERR_ARG
    s.enqueue_monitored(cd.data_ptr())
    # one pending record per handle
    with pytest.raises(_lib.TnsError) as e:
        s.enqueue_monitored(cd.data_ptr())
    assert e.value.code == _lib.TNS_ERR_STATE
    s.synchronize()
    assert np.all(cd.numpy() > 0)
    s.close()
    # a renumbered (general) mesh: the synchronous calls only
    gmesh, _ = cases.renumbered_mesh(mesh, seed=1)
    g = Solver(gmesh, flow, ri)
    with pytest.raises(_lib.TnsError) as e:
        g.upload_async([pinned[m].data_ptr() for m in range(5)])
    assert e.value.code == _lib.TNS_ERR_UNSUPPORTED
    g.close()
