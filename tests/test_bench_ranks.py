"""The multi-rank path of bench.py on CPU (gloo, world size 2): every rank
runs its own replica, the job time is the largest rank's device time, the
whole-job value counts all ranks' cell updates, and the reference arm runs on
rank 0 only."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(times[rank], dist, "cpu")
        out[rank] = (t, bench.replica_value(1000, 10, t, world))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_job_time_is_the_slowest_rank_and_value_counts_all_ranks():
    world, port = 2, _free_port()
    times = [0.25, 0.5]
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, times, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        t, v = res[rank]
        assert t == 0.5
        assert v == pytest.approx(world * 1000 * 10 / 0.5 / 1e9)


def test_single_process_uses_its_own_time():
    assert bench.max_over_ranks(0.3, None, "cpu") == 0.3


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    monkeypatch.setenv("RANK", "1")
    assert bench.run_reference_arm(None) is None
