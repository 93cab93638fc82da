"""Host side of the batched solver: the seeded ramp sweep, the batch manifest format, and
the argument checks tns_batch_create makes before it touches CUDA."""
import ctypes as C

import numpy as np
import pytest

from tnsgpu import _lib, cases, formats


def test_sweep_is_seeded_and_in_range():
    a = cases.ramp_sweep(64, seed=0)
    b = cases.ramp_sweep(64, seed=0)
    c = cases.ramp_sweep(64, seed=1)
    assert a == b and a != c
    assert len(a) == 64 and len({s.name for s in a}) == 64
    for s in a:
        assert 96 <= s.nx <= 512 and s.nx % 32 == 0
        assert 32 <= s.ny <= 192 and s.ny % 32 == 0
        assert 5.0 <= s.angle_deg <= 15.0
        assert 2.0e5 <= s.p0 <= 1.0e6 and 250.0 <= s.t0 <= 400.0
        assert s.amachinit == 0.01
    # the draws cover the ranges
    assert min(s.nx for s in a) <= 160 and max(s.nx for s in a) >= 448
    assert min(s.ny for s in a) == 32 and max(s.ny for s in a) == 192


def test_sweep_case_builds_its_mesh_and_flow():
    s = cases.ramp_sweep(3, seed=0)[2]
    m, f = s.mesh(), s.flow(100)
    assert m.neles == s.nx * s.ny and m.nghosts == 2 * (s.nx + s.ny)
    assert f.p0 == s.p0 and f.t0 == s.t0 and f.istart == 0 and f.niter == 100
    # the ramp rises by tan(angle) * 0.5 m over its second half
    top_wall = m.y[(s.nx) * (s.ny + 1)]
    assert abs(top_wall - 0.5 * np.tan(np.radians(s.angle_deg))) < 1e-9


def test_manifest_round_trip(tmp_path):
    sw = cases.ramp_sweep(5, seed=3)
    p = tmp_path / "batch.in"
    formats.write_manifest(str(p), sw)
    rows = formats.read_manifest(str(p))
    assert len(rows) == 5
    for r, s in zip(rows, sw):
        assert cases.SweepCase(**r) == s


def test_manifest_rejects_short_lines(tmp_path):
    p = tmp_path / "bad.in"
    p.write_text("# name nx ny angle_deg p0 t0 amachinit\nramp 96 32 10.0 2e5\n")
    with pytest.raises(ValueError):
        formats.read_manifest(str(p))


def test_batch_create_checks_arguments_without_gpu():
    L = _lib.load()
    b = C.c_void_p()
    assert L.tns_batch_create(None, 1, C.byref(b)) == _lib.TNS_ERR_ARG
    arr = (C.c_void_p * 2)(None, None)
    rc = L.tns_batch_create(arr, 2, C.byref(b))
    assert rc == _lib.TNS_ERR_ARG
    assert b"null handle" in L.tns_batch_last_error(b)
    L.tns_batch_destroy(b)
    assert L.tns_batch_create(arr, 0, C.byref(b)) == _lib.TNS_ERR_ARG
    assert L.tns_batch_run(None, 1, 0, 0.0, None, None, 0, None, None, None) == _lib.TNS_ERR_ARG
    assert L.tns_batch_launch_count(None) == -1
