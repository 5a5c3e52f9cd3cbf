"""The multi-GPU form of bench.py is replicas (one curve per rank, no collective
on the data path): the job's time is the slowest rank's, and the value is all
ranks' steps over it. Checked here with two gloo ranks on the CPU, plus the
reference arm's rank gating (rank 0 alone works and prints)."""
from __future__ import annotations

import argparse
import datetime
import os
import socket
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
    m = bench.max_over_ranks(ms, dist, "cpu")
    out[rank] = (m, bench.replica_value(4, world, m))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_time_is_the_slowest_rank():
    import torch.multiprocessing as mp

    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0][0] == out[1][0] == 15.0
    assert out[0][1] == pytest.approx(world * 4 / 0.015)
    assert out[1][1] == out[0][1]


def test_single_process_needs_no_group():
    import bench

    assert bench.max_over_ranks(12.5, None, "cpu") == 12.5
    assert bench.replica_value(10, 1, 100.0) == pytest.approx(100.0)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch, capsys):
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    args = argparse.Namespace(V=128, steps=1, warmup=0)
    assert bench.run_reference(args) is None
    assert capsys.readouterr().out == ""
