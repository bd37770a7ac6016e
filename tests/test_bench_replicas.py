"""bench.py --gpus N runs N independent replicas (the path is not sharded): the whole-job
value is the updates of all ranks over the slowest rank's time.  Checked with two gloo
ranks on the CPU."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # Rank r: device time 10 + r ms, 1000 (r + 1) updates; e2e 0.5 (r + 1) s, 800 (r + 1).
        res = bench.replica_totals(dist, "cpu", 10.0 + rank, 1000 * (rank + 1), 0.5 * (rank + 1), 800 * (rank + 1))
        out[rank] = res
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_replica_totals_two_ranks():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        t_max, upd, e2e = out[r]
        assert t_max == 11.0
        assert upd == 3000.0
        assert e2e == pytest.approx(2400.0 / 1.0)


def test_replica_totals_single_process():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.replica_totals(None, "cpu", 5.0, 100, 2.0, 80) == (5.0, 100.0, 40.0)
