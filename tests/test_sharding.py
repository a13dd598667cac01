"""Multi-process sharding logic on CPU (gloo, world size 2)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from tests.helpers import pkg  # noqa: F401  (imports the package path)
import importlib

sharding = importlib.import_module("web-exoplasim_b200.sharding")


@pytest.mark.parametrize("total,world", [(128, 1), (128, 2), (7, 3), (3, 8), (256, 8)])
def test_shards_partition_all_planets(total, world):
    seen = []
    for r in range(world):
        seen.extend(sharding.shard(total, r, world))
    assert seen == list(range(total))
    sizes = [len(sharding.shard(total, r, world)) for r in range(world)]
    assert max(sizes) - min(sizes) <= 1


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
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = sharding.shard(10, rank, world)
        # each rank "times" its own work; the job time is the slowest rank's
        t = sharding.max_over_ranks(1.0 + rank)
        n = sharding.sum_over_ranks(len(mine))
        out.put((rank, list(mine), t, n))
    finally:
        dist.destroy_process_group()


def test_two_rank_reduction_with_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0][1] + results[1][1] == list(range(10))
    assert all(r[2] == 2.0 for r in results)  # max over ranks
    assert all(r[3] == 10 for r in results)   # every planet stepped once
