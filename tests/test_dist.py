"""Multi-process host logic of the N-GPU bench on CPU (gloo, world size 2):
the job's elapsed time is the slowest rank's (max over ranks), ranks meet at
barriers, the whole-job rate of weakly scaled replicas counts every rank's
units, and the reference arm runs on rank 0 only.  The data path has no
collective: ranks process independent burst pairs."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        elapsed = 100.0 + 25.0 * rank  # rank 1 is the slow one
        m = bench.max_over_ranks(elapsed, world)
        bench.barrier(world)
        rate = bench.job_rate(world, 5, 1000, m)
        q.put((rank, m, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_barrier_and_job_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, m, rate in got:
        assert m == 125.0  # every rank sees the slowest rank's time
        assert rate == pytest.approx(2 * 5 * 1000 / 0.125)  # both ranks' units over that time


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    bench.barrier(1)
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.job_rate(1, 10, 50, 1000.0) == 500.0


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    assert bench.run_reference(bench.parse()) is None
    assert capsys.readouterr().out == ""
