"""The replicas' bookkeeping of bench.py on the CPU, as two gloo ranks: the whole-job seconds are
the slowest rank's and the work is summed over the ranks (the same collectives the GPU run makes
over NCCL); the reference arm runs on rank 0 only and the other ranks leave without work."""
import os
import socket
import sys
import types

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
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r: (r + 1) seconds and 10 (r + 1) units of work, twice (device-resident and end to end)
        a = bench.over_ranks(1.0 + rank, 10.0 * (rank + 1), "cpu")
        b = bench.over_ranks(0.5 * (rank + 1), 3.0, "cpu")
        out[rank] = (a, b)
    finally:
        dist.destroy_process_group()


def test_over_ranks_gloo():
    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        (s1, w1), (s2, w2) = res[r]
        assert (s1, w1) == (2.0, 30.0)      # max of 1, 2 s; sum of 10 + 20
        assert (s2, w2) == (1.0, 6.0)


def test_over_ranks_alone():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.over_ranks(1.5, 7.0, "cpu") == (1.5, 7.0)


def test_reference_arm_other_ranks_exit(monkeypatch):
    """Under torchrun the reference arm's rank 0 alone runs and prints; rank 1 returns at once
    (it builds nothing and starts no worker pool)."""
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    a = types.SimpleNamespace(steps=1, warmup=0, workload="c2", inplane=160, gpus=2)
    assert bench.run_reference(a) is None
