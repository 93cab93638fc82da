"""Batched solver (tns_batch_*) against the same cases solved one at a time.

A batch runs the single-case tile code of every kernel phase, launched once over the
tiles of all active cases, so each member's result must equal -- bit for bit -- the
result of that case run alone through tns_run for the same number of iterations, in
both precision modes.  The cases mix mesh sizes (including partial tiles), 2-D and
axisymmetric flows, the global time step (LOCAL=0) and type-6 injection ports.
"""
import numpy as np
import pytest

from tnsgpu import _lib, cases, formats
from tnsgpu.batch import Batch
from tnsgpu.solver import Solver

pytestmark = pytest.mark.gpu


def _axis_sym(mesh):
    mesh.ntype[(mesh.ntype == 5) & (mesh.nside == 1)] = 4
    return mesh


def _case_list():
    ramp_b = cases.ramp_flow(p0=5.0e5, t0=350.0)
    glob = formats.Flow(**{**cases.ramp_flow().__dict__, "local": 0})
    out = [
        ("ramp48x20", cases.ramp_mesh(48, 20), cases.ramp_flow(), "noisy"),
        ("ramp40x36_12deg", cases.ramp_mesh(40, 36, 12.0), ramp_b, "noisy"),
        ("nozzle2d", cases.nozzle_2d_mesh(40, 18), cases.nozzle_2d_flow(), "cold"),
        ("plume_axis_sym", _axis_sym(cases.nozzle_plume_mesh(64, 24)), cases.nozzle_plume_flow(), "cold"),
        ("global_dt", cases.ramp_mesh(40, 16), glob, "noisy"),
        ("port", cases.port_mesh(64, 16), cases.port_flow(), "cold"),
    ]
    return out


def _start(flow, mesh, kind, seed):
    if kind == "noisy":
        return cases.noisy_restart_state(flow, mesh.neles, seed=seed)
    ri = formats.rinit_cold(flow)
    return formats.cold_state(flow, mesh.neles, ri), ri


def _members(precision, pick=None):
    cl = _case_list()
    if pick is not None:
        cl = [cl[k] for k in pick]
    out = []
    for k, (name, mesh, flow, kind) in enumerate(cl):
        c0, ri = _start(flow, mesh, kind, seed=k)
        out.append((name, mesh, flow, c0, ri))
    return out


def _solo(mesh, flow, c0, ri, precision, chunks, monitor=0):
    s = Solver(mesh, flow, ri, precision=precision)
    s.upload(c0)
    rec = []
    for n in chunks:
        if n:
            rec.append(s.run(n, monitor))
    out = s.download(), s.primitives()
    s.close()
    return out, rec


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("precision", [0, 1])
def test_batch_equals_solo_runs(precision, schedule):
    mem = _members(precision)
    solvers = []
    for name, mesh, flow, c0, ri in mem:
        s = Solver(mesh, flow, ri, precision=precision)
        s.upload(c0)
        solvers.append(s)
    b = Batch(solvers, schedule=schedule)
    assert b.schedule == schedule
    # odd then even iteration counts: the mixed path's state parity crosses calls
    r1 = b.run(3, monitor_every=0)
    r2 = b.run(4, monitor_every=2)
    assert list(r1.iterations) == [3] * len(mem) and list(r2.iterations) == [4] * len(mem)
    assert all(len(r) == 2 for r in r2.records)
    for k, (name, mesh, flow, c0, ri) in enumerate(mem):
        (q, prim), rec = _solo(mesh, flow, c0, ri, precision, [3, 4], monitor=2)
        np.testing.assert_array_equal(solvers[k].download(), q, err_msg=name)
        np.testing.assert_array_equal(solvers[k].primitives(), prim, err_msg=name)
        np.testing.assert_array_equal(r2.records[k], rec[1], err_msg=name)
    # members keep working on their own after the batch
    solvers[0].run(1, 0)
    b.close()
    for s in solvers:
        s.close()


def test_masked_case_does_not_move():
    mem = _members(1, pick=[0, 1, 2])
    solvers = [Solver(m, f, ri, precision=1) for _, m, f, _, ri in mem]
    for s, (_, _, _, c0, _) in zip(solvers, mem):
        s.upload(c0)
    b = Batch(solvers)
    b.set_active([1, 0, 1])
    r = b.run(5, monitor_every=0)
    assert list(r.iterations) == [5, 0, 5]
    np.testing.assert_array_equal(solvers[1].download(), mem[1][3])
    b.set_active([1, 1, 1])
    r = b.run(2, monitor_every=0)
    assert list(r.iterations) == [2, 2, 2]
    for k, chunks in ((0, [7]), (1, [2]), (2, [7])):
        _, mesh, flow, c0, ri = mem[k]
        (q, _), _ = _solo(mesh, flow, c0, ri, 1, chunks)
        np.testing.assert_array_equal(solvers[k].download(), q)
    b.close()


def test_convergence_mask_stops_cases_at_their_criterion():
    """stop_ratio masks a case off at the first record with max_k CDIFF_k/REF_k <= ratio;
    each case's state then equals a solo run of the iterations it did."""
    mem = _members(0, pick=[0, 2, 4])
    solvers = [Solver(m, f, ri, precision=0) for _, m, f, _, ri in mem]
    for s, (_, _, _, c0, _) in zip(solvers, mem):
        s.upload(c0)
    b = Batch(solvers)
    # the first-iteration CDIFF of a noisy restart is large, so a loose ratio stops early
    r = b.run(60, monitor_every=5, stop_ratio=0.5)
    assert np.all(r.reference > 0)
    for k, (name, mesh, flow, c0, ri) in enumerate(mem):
        it = int(r.iterations[k])
        assert it % 5 == 0 or it == 60, (name, it)
        recs = r.records[k]
        ratios = np.max(recs / r.reference[k], axis=1)
        if it < 60:
            assert r.active[k] == 0
            assert ratios[-1] <= 0.5 and np.all(ratios[:-1] > 0.5), (name, ratios)
        else:
            assert np.all(ratios > 0.5)
        (q, _), _ = _solo(mesh, flow, c0, ri, 0, [it])
        np.testing.assert_array_equal(solvers[k].download(), q, err_msg=name)
    b.close()


@pytest.mark.parametrize("schedule", [0, 1])
def test_non_finite_case_is_masked_and_others_continue(schedule):
    mem = _members(1, pick=[0, 1])
    solvers = [Solver(m, f, ri, precision=1) for _, m, f, _, ri in mem]
    bad = mem[0][3].copy()
    bad[0, 7] = np.nan  # a NaN density in a restart state: arithmetic only, no indexing
    solvers[0].upload(bad)
    solvers[1].upload(mem[1][3])
    b = Batch(solvers, schedule=schedule)
    with pytest.raises(_lib.TnsError) as e:
        b.run(4, monitor_every=2)
    assert e.value.code == _lib.TNS_ERR_NONFINITE
    r = b.run(4, monitor_every=2, raise_on_failure=False)
    assert r.status[0] == _lib.TNS_ERR_NONFINITE and r.status[1] == _lib.TNS_OK
    assert list(b.active()) == [0, 1]
    _, mesh, flow, c0, ri = mem[1]
    (q, _), _ = _solo(mesh, flow, c0, ri, 1, [8])
    np.testing.assert_array_equal(solvers[1].download(), q)
    # a finite state uploaded again and the case re-activated: it runs and stays finite
    solvers[0].upload(mem[0][3])
    b.set_active([1, 1])
    r = b.run(2, monitor_every=1)
    assert list(r.status) == [0, 0] and list(r.iterations) == [2, 2]
    b.close()


def test_sweep_members_match_solo():
    """Four cases of the seeded ramp sweep (sizes up to 512 x 192), mixed precision."""
    sw = cases.ramp_sweep(64, seed=0)
    pick = [sw[k] for k in (0, 5, 17, 40)]
    solvers, starts = [], []
    for c in pick:
        mesh, flow = c.mesh(), c.flow()
        ri = formats.rinit_cold(flow)
        c0 = formats.cold_state(flow, mesh.neles, ri)
        s = Solver(mesh, flow, ri, precision=1)
        s.upload(c0)
        solvers.append(s)
        starts.append((mesh, flow, c0, ri))
    b = Batch(solvers)
    b.run(20, monitor_every=10)
    for s, (mesh, flow, c0, ri), c in zip(solvers, starts, pick):
        (q, _), _ = _solo(mesh, flow, c0, ri, 1, [20])
        np.testing.assert_array_equal(s.download(), q, err_msg=c.name)
    b.close()


@pytest.mark.parametrize("ti", [4, 16])
def test_tile_height_variants(ti):
    """The TI = 4 and TI = 16 builds: FP64 bit-identical to TI = 8 (same per-cell
    arithmetic), mixed within the mixed path's own FP32 tolerance (its per-tile
    reference flux moves with the tiling)."""
    from tnsgpu import autotune
    assert ti in autotune.available_tile_heights()
    for precision in (0, 1):
        # the port case's C5 is ill-conditioned in the mixed mode (its FP32 envelope is
        # wider than these tolerances); it is checked in FP64 only
        for name, mesh, flow, c0, ri in _members(precision, pick=[0, 3, 5] if precision == 0 else [0, 1, 3]):
            s = Solver(mesh, flow, ri, precision=precision, lib=_lib.variant_path(ti))
            s.upload(c0)
            s.run(5, 0)
            q = s.download()
            s.close()
            (q8, _), _ = _solo(mesh, flow, c0, ri, precision, [5])
            if precision == 0:
                np.testing.assert_array_equal(q, q8, err_msg=f"{name} TI={ti}")
            else:
                rel = np.max(np.abs(q - q8), axis=1) / np.max(np.abs(q8), axis=1)
                assert np.all(rel < np.array([2e-6, 1e-4, 1e-4, 2e-6, 5e-5])), (name, ti, rel)


def test_autotune_batch_picks_a_timed_configuration():
    from tnsgpu import autotune
    mem = _members(1, pick=[0, 1, 2])

    def make(lib):
        out = []
        for _, mesh, flow, c0, ri in mem:
            s = Solver(mesh, flow, ri, precision=1, lib=lib)
            s.upload(c0)
            out.append(s)
        return out

    r = autotune.tune_batch(make, iters=3, warmup=1)
    assert r["ti"] in (4, 8, 16) and r["schedule"] in (0, 1, 2, 3)
    timed = [t for t in r["trials"] if "s_per_iter" in t]
    assert len(timed) == 12 and r["s_per_iter"] == min(t["s_per_iter"] for t in timed)


@pytest.mark.parametrize("precision", [0, 1])
def test_schedule2_iteration_blocks_and_parity_offset(precision):
    """Schedule 2 runs blocks of 8 unmonitored iterations per graph between monitor
    points, and after an odd-length call starts the next at the other state parity
    instead of re-capturing: states and records still equal solo runs bit for bit."""
    mem = _members(precision, pick=[0, 1, 3])
    solvers = [Solver(m, f, ri, precision=precision) for _, m, f, _, ri in mem]
    for s, (_, _, _, c0, _) in zip(solvers, mem):
        s.upload(c0)
    b = Batch(solvers, schedule=2)
    b.run(3, monitor_every=0)
    r = b.run(21, monitor_every=10)
    assert list(r.iterations) == [21] * 3 and all(len(x) == 2 for x in r.records)
    for k, (name, mesh, flow, c0, ri) in enumerate(mem):
        s = Solver(mesh, flow, ri, precision=precision)
        s.upload(c0)
        s.run(3, 0)
        rec = s.run(21, 10)
        np.testing.assert_array_equal(solvers[k].download(), s.download(), err_msg=name)
        np.testing.assert_array_equal(r.records[k], rec, err_msg=name)
        s.close()
    b.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_persistent_schedule_equals_solo_runs(precision):
    """Schedule 3: unmonitored runs of iterations in one cooperative launch (grid
    barriers between the phases), monitored iterations as schedule 0; members equal
    their solo runs bit for bit, across calls of odd and even length."""
    mem = _members(precision, pick=[0, 1, 2, 3])  # LOCAL=1, no port
    solvers = []
    for name, mesh, flow, c0, ri in mem:
        s = Solver(mesh, flow, ri, precision=precision)
        s.upload(c0)
        solvers.append(s)
    b = Batch(solvers, schedule=3)
    assert b.schedule == 3
    l0 = b.launch_count()
    r1 = b.run(37, monitor_every=10)
    r2 = b.run(4, monitor_every=0)
    assert list(r1.iterations) == [37] * len(mem) and list(r2.iterations) == [4] * len(mem)
    for k, (name, mesh, flow, c0, ri) in enumerate(mem):
        (q, prim), rec = _solo(mesh, flow, c0, ri, precision, [37, 4], monitor=10)
        np.testing.assert_array_equal(solvers[k].download(), q, err_msg=name)
        np.testing.assert_array_equal(solvers[k].primitives(), prim, err_msg=name)
        np.testing.assert_array_equal(r1.records[k], rec[0], err_msg=name)
    # 41 iterations, 3 of them monitored: a handful of persistent launches, not 6 a case
    assert b.launch_count() - l0 < 40
    b.close()
    for s in solvers:
        s.close()


def test_persistent_schedule_refuses_what_it_cannot_run():
    for pick in ([4], [5]):  # LOCAL=0; a type-6 port
        mem = _members(0, pick=pick)
        solvers = []
        for name, mesh, flow, c0, ri in mem:
            s = Solver(mesh, flow, ri)
            s.upload(c0)
            solvers.append(s)
        with pytest.raises(_lib.TnsError) as e:
            Batch(solvers, schedule=3)
        assert "schedule 3" in str(e.value)
        for s in solvers:
            s.close()



@pytest.mark.parametrize("precision", [0, 1])
def test_batch_with_general_meshes_equals_solo_runs(precision):
    """A batch holding general-mesh cases (ids shuffled, faces rotated: no tile table)
    beside structured ones runs every case through its own iteration (schedules 1 and
    2), bit-identical to the cases run alone; the tile-table schedules are refused."""
    mem = _members(precision, pick=[0, 2, 4])
    runs = []
    for k, (name, mesh, flow, c0, ri) in enumerate(mem):
        if k != 1:  # the nozzle stays one structured block
            mesh, perm = cases.renumbered_mesh(mesh, seed=11 + k)
            q = np.empty_like(c0)
            q[:, perm] = c0
            c0 = q
        runs.append((name, mesh, flow, c0, ri))
    solvers = []
    for name, mesh, flow, c0, ri in runs:
        s = Solver(mesh, flow, ri, precision=precision)
        s.upload(c0)
        solvers.append(s)
    b = Batch(solvers)
    assert b.schedule == 2
    for bad in (0, 3):
        with pytest.raises(_lib.TnsError) as e:
            b.schedule = bad
        assert e.value.code == _lib.TNS_ERR_UNSUPPORTED
    r1 = b.run(3, monitor_every=0)
    b.schedule = 1
    r2 = b.run(10, monitor_every=5)
    assert list(r1.iterations) == [3] * len(runs) and list(r2.iterations) == [10] * len(runs)
    for k, (name, mesh, flow, c0, ri) in enumerate(runs):
        (q, prim), rec = _solo(mesh, flow, c0, ri, precision, [3, 10], monitor=5)
        np.testing.assert_array_equal(solvers[k].download(), q, err_msg=name)
        np.testing.assert_array_equal(solvers[k].primitives(), prim, err_msg=name)
        np.testing.assert_array_equal(r2.records[k], rec[1], err_msg=name)
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.parametrize("schedule", [0, 1, 2, 3])
@pytest.mark.parametrize("precision", [0, 1])
def test_prepare_captures_without_running(precision, schedule):
    """tns_prepare / tns_batch_prepare capture every graph ahead of the runs: they launch
    nothing (launch counts unchanged, states unchanged), a second call is a no-op, and
    the runs after them equal solo runs bit for bit, across calls of odd and even
    length (both state parities)."""
    mem = _members(precision, pick=[0, 1, 3])  # LOCAL=1, no port: every schedule runs them
    solvers = []
    for name, mesh, flow, c0, ri in mem:
        s = Solver(mesh, flow, ri, precision=precision)
        s.upload(c0)
        solvers.append(s)
    b = Batch(solvers, schedule=schedule)
    l0 = b.launch_count()
    b.prepare()
    b.prepare()
    assert b.launch_count() == l0
    for s, (name, _, _, c0, _) in zip(solvers, mem):
        np.testing.assert_array_equal(s.download(), c0, err_msg=name)
    r1 = b.run(3, monitor_every=0)
    r2 = b.run(21, monitor_every=10)
    assert list(r1.iterations) == [3] * len(mem) and list(r2.iterations) == [21] * len(mem)
    for k, (name, mesh, flow, c0, ri) in enumerate(mem):
        s = Solver(mesh, flow, ri, precision=precision)
        s.upload(c0)
        n0 = s.launch_count()
        s.prepare()
        s.prepare()
        assert s.launch_count() == n0, name
        np.testing.assert_array_equal(s.download(), c0, err_msg=name)
        s.run(3, 0)
        rec = s.run(21, 10)
        np.testing.assert_array_equal(solvers[k].download(), s.download(), err_msg=name)
        np.testing.assert_array_equal(r2.records[k], rec, err_msg=name)
        s.close()
    b.close()
    for s in solvers:
        s.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_sweep_cli_compare_on_a_small_sweep(precision):
    """tnsgpu.sweep.compare (the sweep CLI) on four cases of the seeded sweep: the batched
    and sequential arms agree bit for bit (same build, no tuning) and both report their
    times."""
    from tnsgpu import sweep
    r = sweep.compare(ncases=4, niter=30, stop_ratio=1.0e-5, monitor=10, seed=0, precision=precision,
                      tune=False)
    assert r["iterations_equal"] and r["states_bitwise_equal"] and r["state_rel_diff_max"] == 0.0
    assert r["iterations_min_max"] == [30, 30]
    assert r["batched_s"] > 0 and r["sequential_s"] > 0 and r["batch_launches"] > 0
