"""The multi-GPU form of the benchmark is replicas: each rank runs the whole per-GPU workload, the job's time is the
slowest rank's, and the job's rate counts every rank's units. The host side of that, on two gloo ranks on the CPU."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out) -> None:
    import datetime

    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 + 25.0 * rank  # rank 1 is the slow one
        job_ms = bench.max_over_ranks_of(local_ms, world, torch.device("cpu"))
        out.put((rank, job_ms, bench.job_rate(1e9, 4, world, job_ms)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank_and_count_every_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [125.0, 125.0]
    # 4 steps of 1e9 units on each of 2 ranks in 125 ms
    assert res[0][2] == pytest.approx(2 * 4e9 / 0.125)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    """Under torchrun the reference arm's other ranks exit at once without work or output."""
    import argparse

    monkeypatch.setenv("RANK", "1")
    bench.run_reference_arm(argparse.Namespace(workload="mixed", steps=1, warmup=0, gpus=2))
    assert capsys.readouterr().out == ""
