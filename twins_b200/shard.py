"""Worlds across GPUs: one process per GPU, worlds partitioned by their estimated work, no
collective on the data path (worlds never exchange frames). Results are gathered on the host.

    shard(worlds, rank, size)   the indices of the worlds rank `rank` runs (balanced greedy)
    aggregate(ms, events, dist) max device time and summed events over ranks (timing rule:
                                max over ranks)
"""
from __future__ import annotations

from typing import Optional, Sequence

MSS = 1460


def work_of(world) -> float:
    """A world's estimated work: its segments (bytes / MSS) times a path-length factor
    (hops of a FatTree or leaf-spine path are at most 4 switches)."""
    f = world.flows
    segs = float((f.size // MSS + 1).sum())
    return segs * 8.0 + len(f)


def shard(worlds: Sequence, rank: int, size: int) -> list[int]:
    """Longest-processing-time greedy: worlds by decreasing work, each to the least-loaded rank;
    deterministic on every rank (ties by world index, then rank)."""
    if size < 1 or not 0 <= rank < size:
        raise ValueError("rank out of range")
    order = sorted(range(len(worlds)), key=lambda i: (-work_of(worlds[i]), i))
    load = [0.0] * size
    owner = [0] * len(worlds)
    for i in order:
        r = min(range(size), key=lambda j: (load[j], j))
        owner[i] = r
        load[r] += work_of(worlds[i])
    return [i for i in range(len(worlds)) if owner[i] == rank]


def aggregate(ms: float, events: float, dist=None, device: Optional[str] = None) -> tuple[float, float]:
    """(max of ms over ranks, sum of events over ranks); without a process group, the inputs."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return ms, events
    import torch
    t = torch.tensor([ms, events], dtype=torch.float64, device=device or "cpu")
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    tot = t.clone()
    dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return float(mx[0]), float(tot[1])
