"""The multi-GPU path of the benchmark on CPU: two `gloo` ranks (world size 2)
run the same rank-level logic the NCCL ranks run -- distinct seeded batches
per replica, and whole-job throughput from the max elapsed time over ranks."""
import os
import socket

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 * (rank + 1)  # the second replica is the slow one
        ms, value = bench.aggregate_over_ranks(dist, local_ms, "cpu", 1000, 4, world)
        x, e, m = bench.make_inputs(64, 8, seed=bench.replica_seed(rank))
        out[rank] = (ms, value, x.tobytes())
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo():
    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    for r in range(world):
        ms, value, _ = res[r]
        assert ms == pytest.approx(200.0)                       # max over ranks, seen by every rank
        assert value == pytest.approx(2 * 1000 * 4 / 0.2)      # all ranks' instances / slowest time
    assert res[0][2] != res[1][2]                               # each replica has its own batch
