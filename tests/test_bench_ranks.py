"""The multi-replica host logic of bench.py (one process per GPU, no data-path collective):
the job's step time is the max over ranks and its rate counts every rank's cells; only
rank 0 runs and prints the reference arm.  Two gloo ranks on the CPU."""

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
    sys.path.insert(0, ROOT)
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks_of(10.0 + 5.0 * rank, dist, "cpu")  # rank 1 is the slow one
        out[rank] = (ms, bench.job_throughput(1000, world, ms))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_max_over_ranks():
    world = 2
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        ms, rate = out[r]
        assert ms == 15.0
        assert rate == pytest.approx(1000 * 2 / 0.015)


def test_single_process_keeps_its_own_time():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks_of(12.5, None, "cpu") == 12.5


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class A:
        steps, warmup, gpus = 1, 0, 2

    assert bench.run_reference(A()) is None
    assert capsys.readouterr().out == ""


def test_reference_arm_prints_the_contract_line(monkeypatch, capsys):
    """The CPU reference arm: one JSON line with the metric, its unit and direction, the
    CPU baseline it measured and an e2e entry that moves no bytes."""
    import json

    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "0")
    monkeypatch.setenv("WORLD_SIZE", "1")

    class A:
        steps, warmup, gpus = 1, 0, 1

    bench.run_reference(A())
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC
    assert line["unit"] == "cell-iters/s" and line["higher_is_better"] is True and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["cpu_baseline"]["value"] == line["value"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["config"]["workload"].startswith("C2: 500000 cells")
