"""Host logic of the multi-GPU bench path on CPU: world size 2 over gloo.

The solver path does not shard, so `bench.py --gpus N` runs N independent
replicas; the only collectives are a start barrier and the max of the ranks'
device times. These tests run that aggregation in two gloo processes and check
the whole-job rate, and that the reference arm prints on rank 0 only."""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

from tests.conftest import ROOT

sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, times, q):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        tmax = bench.max_over_ranks(times[rank], world)
        q.put((rank, tmax, bench.whole_job_rate(world, 20, tmax)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_time_is_max_over_ranks_and_rate_counts_every_replica():
    world, port = 2, _free_port()
    times = [812.5, 1000.0]  # ms of 20 steps on each rank
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, times, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(world))
    for rank, tmax, rate in out:
        assert tmax == 1000.0
        assert rate == pytest.approx(2 * 1000.0 * 20 / 1000.0)  # 40 whole-job steps/s


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.whole_job_rate(1, 10, 500.0) == pytest.approx(20.0)


def test_reference_arm_prints_on_rank_0_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                                      "--warmup", "0"])
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.main()
    assert buf.getvalue() == ""
