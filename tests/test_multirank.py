"""The N>1 host logic of bench.py on CPU: world-size-2 gloo process groups.

With N GPUs every rank renders its own frame (replicas, weak scaling) and the
step time is the maximum over ranks; the reference arm runs on rank 0 only.
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        import bench
        step_ms = [12.5, 17.25][rank]
        results[rank] = (bench.max_over_ranks(step_ms, world, "cpu"), bench.max_over_ranks(1.0, 1, "cpu"))
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        results = m.dict()
        mp.start_processes(_worker, args=(2, free_port(), results), nprocs=2, join=True, start_method="spawn")
        assert results[0] == (17.25, 1.0) and results[1] == (17.25, 1.0)


def test_reference_arm_does_no_work_on_other_ranks(monkeypatch):
    sys.path.insert(0, str(ROOT))
    import bench
    monkeypatch.setenv("RANK", "1")
    # rank 1 returns before building any scene or touching the oracle
    assert bench.run_reference(type("A", (), {"paths": 0, "size": 0, "steps": 1, "warmup": 0})()) is None
