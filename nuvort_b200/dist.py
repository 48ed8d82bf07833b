"""Multi-GPU helpers.  One process per GPU (torchrun).

* Independent systems shard across ranks (`shard_systems`) with no data-path collective;
  the only collectives are a barrier around timed regions and the reductions of per-rank
  timings (max) and work (sum).
* One tangle splits its velocity pass over the ranks (`TangleSplit`): every rank keeps the
  whole state and builds the same tree; each computes the targets of its range of the walk
  order, the ranges' velocities are all-gathered, and every rank finishes the step (AB3
  update and topology) on the full field, so that all ranks hold the one-GPU state, bit for
  bit, after every step.
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


WARP = 32  # walk positions per warp of the tree walks


def split_ranges(live: int, world: int) -> List[tuple]:
    """Walk-position ranges [lo, hi) of the ranks: positions 1 .. live (the live points in the
    walk order) in near-equal contiguous parts of whole warps (every end but live + 1 at
    1 + a multiple of 32), so that no warp of the mixed walk is cut in two."""
    warps = -(-live // WARP)
    out = []
    for r in range(world):
        lo = min(1 + (r * warps) // world * WARP, live + 1)
        hi = min(1 + ((r + 1) * warps) // world * WARP, live + 1)
        out.append((lo, hi))
    return out


def walk_range(lo: int, hi: int, cap: int) -> tuple:
    """The nv_set_walk_range arguments for positions [lo, hi) of split_ranges: an end at
    live + 1 off a warp boundary becomes cap + 1 (the positions past live hold no target),
    and an empty range (1, 1)."""
    if hi <= lo:
        return 1, 1
    return lo, hi if (hi - 1) % WARP == 0 else cap + 1


class TangleSplit:
    """A step of one tangle (system `sys` of `handle`) with its velocity pass split over the
    ranks of `dist` (torch.distributed, initialised; NCCL with CUDA tensors or gloo with CPU
    ones).  `device` is where the exchange buffers live ("cuda" for the library's own
    velocities, which nv_velocity_pack/unpack read and write in device memory)."""

    def __init__(self, handle, sys: int, dist, device: str = "cuda"):
        self.h = handle
        self.sys = sys
        self.dist = dist
        self.rank = dist.get_rank()
        self.world = dist.get_world_size()
        self.device = device

    def step(self):
        import torch
        live = int(self.h.counters(self.sys).live)  # the same on every rank
        # every rank checks that: ranks that disagreed would size the all-gather differently
        # and wait on one another instead of failing
        agree = torch.tensor([live, -live], dtype=torch.int64, device=self.device)
        self.dist.all_reduce(agree, op=self.dist.ReduceOp.MAX)
        if int(agree[0]) != -int(agree[1]):
            raise RuntimeError(f"TangleSplit: the ranks' live counts differ (from {-int(agree[1])} to "
                               f"{int(agree[0])}); their states have diverged")
        ranges = split_ranges(live, self.world)
        lo, hi = ranges[self.rank]
        self.h.set_walk_range(self.sys, *walk_range(lo, hi, self.h.capacity[self.sys]))
        self.h.step_velocity()
        width = max(b - a for a, b in ranges)
        # uninitialised: the rows past hi - lo are sent but never read, and no fill kernel on
        # torch's stream races the library's pack on its own stream
        mine = torch.empty((max(width, 1), 3), dtype=torch.float64, device=self.device)
        self.h.velocity_pack(self.sys, lo, hi - lo, mine.data_ptr())
        parts = [torch.empty_like(mine) for _ in range(self.world)]
        if self.device != "cpu":
            torch.cuda.synchronize()
        self.dist.all_gather(parts, mine)
        if self.device != "cpu":
            torch.cuda.synchronize()
        for r, (a, b) in enumerate(ranges):
            if r != self.rank and b > a:
                self.h.velocity_unpack(self.sys, a, b - a, parts[r].data_ptr())
        self.h.step_finish()
