"""Multi-GPU helpers: independent systems shard across ranks with no data-path collective.

One process per GPU (torchrun).  The only collectives are for measurement and bookkeeping:
a barrier around timed regions and the reductions of per-rank timings (max) and work (sum).
"""
from __future__ import annotations

from typing import List, Sequence


def shard_systems(counts: Sequence[int], world: int, rank: int) -> List[int]:
    """Indices of the systems rank `rank` owns: greedy balance of the N^2 work proxy
    (largest systems first, each to the currently lightest rank; ties to the lowest rank)."""
    load = [0.0] * world
    owner = [0] * len(counts)
    for s in sorted(range(len(counts)), key=lambda s: (-counts[s], s)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[s] = r
        load[r] += float(counts[s]) ** 2
    return [s for s in range(len(counts)) if owner[s] == rank]


def reduce_max_sum(dist, device, maxes: Sequence[float], sums: Sequence[float]):
    """All-reduce: element-wise max of `maxes` and sum of `sums` over ranks (identity when
    dist is None).  Every rank makes the same calls in the same order."""
    import torch
    mx = torch.tensor(list(maxes), dtype=torch.float64, device=device)
    sm = torch.tensor(list(sums), dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return [float(v) for v in mx], [float(v) for v in sm]
