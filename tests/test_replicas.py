"""Multi-GPU bench path on CPU ranks: the single-mesh solve does not shard, so N ranks run N
independent replicas and the only collective is the timing reduction.  Two `gloo` ranks (no GPU)
check that the bench's reduction returns the slowest rank's times on every rank and that the
whole-job throughput is ranks x steps over that time."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from tests.conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        ms = [100.0 + 10.0 * rank, 120.0 - 5.0 * rank]        # (value leg, e2e leg) of this rank
        out[rank] = bench.max_over_ranks(dist, ms, "cpu")
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replica_timing_reduction_two_ranks():
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        results = dict(out)
    assert results[0] == results[1] == [110.0, 120.0]
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.replica_throughput(world, 3, 110.0) == pytest.approx(2 * 3 / 0.110)
    assert bench.max_over_ranks(None, [1.5, 2.5], "cpu") == [1.5, 2.5]
