"""One process per GPU: rank layout, work sharding and timing over ranks.

The CA path shards without a data-path collective in two ways: independent
replicas of a domain (weak scaling) and an ensemble of independent domains
dealt to the ranks (strong scaling).  Ranks exchange only the timing (the
max over ranks) and small summaries.  The helpers work with any
torch.distributed backend (NCCL on the GPUs, gloo for CPU tests).
"""
from __future__ import annotations

import os


def dist_env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the launcher's environment."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def shard(n: int, rank: int, world: int) -> list[int]:
    """Items of an n-item ensemble this rank owns: i with i mod world == rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank layout")
    return list(range(rank, n, world))


def shard_balanced(sizes: list[int], world: int) -> list[list[int]]:
    """Deal items to ranks largest first, each to the least-loaded rank
    (ties to the lowest rank): every rank gets a list of item indices."""
    if world < 1:
        raise ValueError("bad world size")
    loads = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += sizes[i]
    for lst in out:
        lst.sort()
    return out


def max_over_ranks(x: float, device=None) -> float:
    """x maximised over the ranks of the default process group (x itself
    without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
