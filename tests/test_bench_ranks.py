"""bench.py's multi-rank plumbing on CPU (the replicas-only N-GPU path): two gloo
ranks, as torchrun would start them, agree on the slowest rank's time and on the
whole-job rate; the reference arm does its work on rank 0 only."""

import os
import socket
import sys
from pathlib import Path
from types import SimpleNamespace

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    from datetime import timedelta

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench

    # rank r took 10 (r + 1) ms for 256 clips; a second collective in the same order on every rank
    ms = bench.max_over_ranks(10.0 * (rank + 1), world, dist, "cpu")
    ms2 = bench.max_over_ranks(5.0 - rank, world, dist, "cpu")
    q.put((rank, ms, bench.whole_job_rate(world, 256, ms), ms2))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate, ms2 in out:
        assert ms == 20.0 and ms2 == 5.0
        assert rate == pytest.approx(2 * 256 / 0.020)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(7.5, 1, None, "cpu") == 7.5
    assert bench.whole_job_rate(1, 256, 100.0) == pytest.approx(2560.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    called = []
    monkeypatch.setattr(bench, "_cpu_clip_solves", lambda *a, **k: called.append(1) or (1, 1.0, 1))
    assert bench.run_reference(SimpleNamespace(warmup=1, steps=1)) == 0
    assert not called
