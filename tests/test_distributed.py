"""Rank layout, sharding and timing over ranks (mumatscale_b200.distributed),
as two gloo processes on the CPU."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from mumatscale_b200 import distributed as D


def test_shard_round_robin():
    parts = [D.shard(10, r, 3) for r in range(3)]
    assert parts == [[0, 3, 6, 9], [1, 4, 7], [2, 5, 8]]
    with pytest.raises(ValueError):
        D.shard(10, 3, 3)


def test_shard_balanced_partitions():
    sizes = [5, 1, 9, 3, 3, 7, 2, 8]
    parts = D.shard_balanced(sizes, 3)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    loads = [sum(sizes[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank: int, world: int, port: int, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=60))
    try:
        ws, r, _ = D.dist_env()
        from mumatscale_b200 import workloads as W
        sizes = []
        for deck in W.ensemble(64):
            dims = [int(v) for v in deck.split("NCellsPerSB")[1].split("\n")[0].split()]
            sizes.append(dims[0] * dims[1] * dims[2])
        mine = D.shard_balanced(sizes, ws)[r]
        cells = sum(sizes[i] for i in mine)
        gathered = [None] * ws
        dist.all_gather_object(gathered, mine)
        total = D.sum_over_ranks(cells)
        slowest = D.max_over_ranks(float(r + 1))
        q.put((r, gathered, total, sum(sizes), slowest))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_the_ensemble():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, gathered, total, want, slowest in results:
        flat = sorted(i for part in gathered for i in part)
        assert flat == list(range(64))
        assert not set(gathered[0]) & set(gathered[1])
        assert total == want
        assert slowest == 2.0
