"""The multi-rank (N>1) path of bench.py on CPU: two gloo ranks, the way the
driver launches one process per GPU.  The path shards by query with no data
collective; what crosses ranks is the slowest rank's step time."""
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
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    # each rank reports a different step time; every rank must see the maximum
    got = bench.max_over_ranks(10.0 + rank * 5.0, world, "cpu")
    out[rank] = got
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(out) == {0: 15.0, 1: 15.0}


def _shard_rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    mine = bench.shard(range(1000), rank, world)
    every = [None] * world
    dist.all_gather_object(every, mine)
    out[rank] = every
    dist.barrier()
    dist.destroy_process_group()


def test_batch_is_split_by_query_across_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    every = out[0]
    assert out[1] == every
    # each query lands on exactly one rank, and the ranks' shares differ by at most one
    assert sorted(x for part in every for x in part) == list(range(1000))
    assert abs(len(every[0]) - len(every[1])) <= 1


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
