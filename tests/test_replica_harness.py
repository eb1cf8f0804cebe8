"""The multi-GPU harness of bench.py runs independent replicas: the only
exchange is the max over ranks of each timing.  Checked here with two gloo
ranks on the CPU (no GPU): every rank gets the largest value, and the
reference arm does no work on ranks other than 0."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        v = bench.max_over_ranks(dist, 10.0 + rank, device="cpu")
        w = bench.max_over_ranks(dist, 5.0 - rank, device="cpu")
        out[rank] = (v, w)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        assert dict(out) == {0: (11.0, 5.0), 1: (11.0, 5.0)}


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(None, 3.5) == 3.5


def test_reference_arm_skips_nonzero_ranks(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench

    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "build_case", lambda: called.append(1))
    bench.run_reference(None)
    assert called == []
