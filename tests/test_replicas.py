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


def _tube_rank(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        specs = bench.c5_specs()
        part = bench.tube_part(specs, world, rank)
        # each rank reports a metric of its own tubes only; the gather puts them in tube order everywhere
        metrics = [{"tube": k, "rank": rank, "elements": specs[k].elements} for k in part]
        out[rank] = (part, bench.gather_tube_metrics(dist, part, metrics))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_batched_tubes_partition_and_gather_two_ranks():
    """The batched-tube workload on two ranks: each rank's tubes come from the same seeded specs and the
    same greedy packing, the parts are disjoint and cover all 64 tubes with balanced cost (within the
    longest-first bound 4/3 of the optimum), and the per-tube metrics gathered over gloo arrive on every
    rank complete and in tube order."""
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_tube_rank, args=(world, _free_port(), out), nprocs=world, join=True)
        results = dict(out)
    sys.path.insert(0, str(ROOT))
    import bench
    from tubularflowiga_b200 import meshgen
    specs = bench.c5_specs()
    parts = [results[r][0] for r in range(world)]
    assert sorted(parts[0] + parts[1]) == list(range(len(specs)))
    assert not set(parts[0]) & set(parts[1])
    costs = [meshgen.tube_cost(s) for s in specs]
    loads = [sum(costs[k] for k in p) for p in parts]
    assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs))
    for r in range(world):
        gathered = results[r][1]
        assert [m["tube"] for m in gathered] == list(range(len(specs)))
        assert all(m["rank"] == (0 if m["tube"] in parts[0] else 1) for m in gathered)
    assert sum(s.elements for s in specs) > 500000 and min(s.elements for s in specs) >= 900
    assert sum(s.curvature_radius > 0 for s in specs) > 16
