"""The multi-GPU plumbing of the benchmark (independent replicas, no data-path collective) on CPU
ranks: world size 2 over gloo.  Every rank meets the others at the timing barriers, takes the
slowest rank's time, and the whole-job rate counts the nodes of every replica; the reference arm
runs on rank 0 only."""
import json
import multiprocessing as mp
import os
import socket

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench.barrier(dist)
        ms = bench.max_over_ranks(dist, 100.0 + 25.0 * rank)  # rank 1 is the slow one
        bench.barrier(dist)
        seconds = bench.max_over_ranks(dist, 0.5 - 0.1 * rank)
        out.put((rank, ms, seconds, bench.whole_job_mlups(world, 1000, 10, ms / 1e3)))
    finally:
        dist.destroy_process_group()


def test_replicas_take_the_slowest_rank_and_count_every_replica():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = sorted(out.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, seconds, rate in results:
        assert ms == 125.0
        assert seconds == 0.5
        # 2 replicas x 1000 nodes x 10 steps in 0.125 s
        assert rate == pytest.approx(2 * 1000 * 10 / 0.125 / 1e6)


def test_single_process_needs_no_process_group():
    import bench
    assert bench.dist_init(1)[:2] == (0, 1)
    assert bench.max_over_ranks(None, 3.5) == 3.5
    assert bench.whole_job_mlups(1, 256 ** 3, 500, 2.0) == pytest.approx(256 ** 3 * 500 / 2.0 / 1e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import argparse

    import bench
    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "cpu_baseline_sample", lambda **kw: called.append(kw))
    args = argparse.Namespace(gpus=2, steps=3, warmup=3)
    assert bench.run_reference_arm(args) == 0
    assert not called and capsys.readouterr().out == ""

    monkeypatch.setenv("RANK", "0")
    monkeypatch.setattr(bench, "cpu_baseline_sample",
                        lambda **kw: {"value": 1.5, "unit": "MLUPS", "cores": kw["processes"], "kind": "reference",
                                      "sample": "stub"})
    assert bench.run_reference_arm(args) == 0
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference" and line["value"] == 1.5 and line["n_gpus"] == 2
    assert line["e2e"] == {"value": 1.5, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
