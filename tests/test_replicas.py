"""bench.py --gpus N runs N independent replicas (the path has no exchange step on one
mesh): every rank times its own replica, the job takes the slowest rank's time, and the
whole-job rate is N * cells / that time.  These run the rank logic as two gloo
processes on the CPU; the reference arm prints from rank 0 only."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(times[rank], world, torch, "cpu")
        out[rank] = (t, bench.replica_rate(1000, t, world))
    finally:
        torch.distributed.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world = 2
    times = [0.25, 0.4]
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), times, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (0.4, 2 * 1000 / 0.4)


def test_single_rank_is_unchanged():
    assert bench.max_over_ranks(0.3, 1, torch, "cpu") == 0.3
    assert bench.replica_rate(393216, 0.5, 1) == 393216 / 0.5


@pytest.mark.parametrize("rank,prints", [(0, True), (1, False)])
def test_reference_arm_prints_from_rank_zero_only(rank, prints):
    env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK=str(rank))
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3", "--case", "ramp_192x64"],
                       env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    if prints:
        line = json.loads(lines[-1])
        assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    else:
        assert lines == []
