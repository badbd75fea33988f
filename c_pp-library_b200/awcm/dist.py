"""Multi-GPU plumbing of the AWCM path: one process per GPU, no data-path collective.

A single AWCM instance is not split across GPUs (its level-sequential mask passes would need a
halo exchange per pass); N GPUs run N replicas of an instance, or share a batch of independent
1D instances.  The only cross-rank traffic is the end-of-run timing/stats reduction below,
over torch.distributed (NCCL on GPUs, gloo on the CPU tests).
"""
from __future__ import annotations

from typing import Sequence


def shard_instances(sizes: Sequence[int], rank: int, world: int) -> list[int]:
    """Instance indices owned by `rank`: greedy largest-first assignment to the least-loaded rank,
    so every rank gets a similar number of points.  Deterministic; the shards partition range(n)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    load = [0] * world
    owner = [0] * len(sizes)
    for k in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda r: (load[r], r))
        owner[k] = r
        load[r] += sizes[k]
    return [k for k in range(len(sizes)) if owner[k] == rank]


def reduce_run(elapsed_ms: float, updates: float, device=None) -> tuple[float, float]:
    """(max over ranks of the device time, sum over ranks of the updates); identity when not
    distributed."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return elapsed_ms, updates
    t = torch.tensor([elapsed_ms], dtype=torch.float64, device=device)
    u = torch.tensor([updates], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(u, op=dist.ReduceOp.SUM)
    return float(t.item()), float(u.item())
