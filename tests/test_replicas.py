"""The multi-GPU path of bench.py is replicas: every rank advances its own
planetesimal and the job's time is the slowest rank's.  Its host-side logic
(barrier, max over ranks, whole-job rate, rank-0-only reference arm) runs
here as two gloo ranks on the CPU."""
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


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(world)
        ms = 100.0 + 50.0 * rank           # rank 1 is the slow one
        out[rank] = (bench.max_over_ranks(ms, world), bench.job_rate(10, ms, world))
        bench.barrier(world)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_time_the_job_by_the_slowest_rank():
    world, port = 2, _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, port, out), nprocs=world, join=True,
                           start_method="spawn")
        res = dict(out)
    for r in range(world):
        slowest, rate = res[r]
        assert slowest == 150.0
        assert rate == pytest.approx(2 * 10 / 0.150)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    args = bench.argparse.Namespace(gpus=2, steps=2, warmup=1, workload=bench.WORKLOAD)
    assert bench.run_reference(args) == 0
    assert capsys.readouterr().out == ""
