"""The multi-rank path on CPU: two gloo ranks shard an ensemble and reduce their timings."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from nuvort_b200.dist import reduce_max_sum, shard_systems


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    counts = [500, 20000, 1200, 7000, 300, 15000, 900]
    mine = shard_systems(counts, world, rank)
    work = float(sum(counts[s] for s in mine))
    step_ms = 10.0 + 5.0 * rank
    mx, sm = reduce_max_sum(dist, "cpu", [step_ms], [work, 1.0])
    q.put((rank, mine, mx, sm))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, mx0, sm0), (r1, m1, mx1, sm1) = res
    assert sorted(m0 + m1) == list(range(7)) and not set(m0) & set(m1)
    assert mx0 == mx1 == [15.0]
    counts = [500, 20000, 1200, 7000, 300, 15000, 900]
    assert sm0 == sm1 == [float(sum(counts)), 2.0]


def test_shard_balances_quadratic_work():
    counts = [20000, 15000, 12000, 9000, 3000, 1000]
    loads = [sum(counts[s] ** 2 for s in shard_systems(counts, 3, r)) for r in range(3)]
    # greedy longest-first: no rank exceeds the largest system or 4/3 of the mean load
    assert max(loads) <= max(max(c ** 2 for c in counts), 4 / 3 * sum(loads) / 3)
    assert shard_systems(counts, 1, 0) == list(range(6))


def _bench_worker(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    params, states, cfg = bench.workload("ensemble512", rank, crossover=3000, world=world)
    mine = sorted((st.pcount, round(p.alpha[0], 12)) for p, st in zip(params, states))
    _, (pts,) = reduce_max_sum(dist, "cpu", [0.0], [float(sum(st.pcount for st in states))])
    q.put((rank, mine, pts, cfg["points"]))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_ensemble_split_over_two_gloo_ranks():
    # bench.py --gpus 2 splits ONE ensemble: the two ranks' systems reassemble it exactly
    # (no system twice, none lost) and the summed points are the whole ensemble's
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    params, states, cfg = bench.workload("ensemble512", 0, crossover=3000, world=1)
    whole = sorted((st.pcount, round(p.alpha[0], 12)) for p, st in zip(params, states))
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, m0, pts0, tot0), (_, m1, pts1, tot1) = res
    assert len(m0) > 0 and len(m1) > 0
    assert sorted(m0 + m1) == whole
    assert pts0 == pts1 == float(sum(st.pcount for st in states)) == tot0 == tot1 == cfg["points"]


class _FakeTangle:
    """Stands in for a handle holding one tangle on CPU: a walk order (perm), a velocity
    field that the 'velocity pass' fills only on the walk range, and the pack/unpack and
    step halves of the C ABI, with host pointers in place of device ones."""

    def __init__(self, n, seed):
        import numpy as np
        rng = np.random.default_rng(seed)
        self.n = n
        self.perm = np.concatenate([[0], 1 + rng.permutation(n)])  # position q -> slot
        self.truth = rng.standard_normal((n + 1, 3))                  # the full field
        self.u = np.zeros((n + 1, 3))
        self.lo, self.hi = 1, n + 1
        self.capacity = [n + 64]
        self.finished = None

    class _C:
        def __init__(self, live):
            self.live = live

    def counters(self, sys):
        return self._C(self.n)

    def set_walk_range(self, sys, lo, hi):
        # the library's rule: ends on warp boundaries, or hi = cap + 1
        assert 1 <= lo <= hi <= self.capacity[0] + 1 and (lo - 1) % 32 == 0
        assert (hi - 1) % 32 == 0 or hi == self.capacity[0] + 1
        self.lo, self.hi = lo, hi

    def step_velocity(self):
        self.u[:] = 0.0
        for q in range(self.lo, min(self.hi, self.n + 1)):
            self.u[self.perm[q]] = self.truth[self.perm[q]]

    def _view(self, ptr, count):
        import ctypes
        import numpy as np
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_double)), shape=(count, 3))

    def velocity_pack(self, sys, lo, count, ptr):
        v = self._view(ptr, count)
        for i in range(count):
            v[i] = self.u[self.perm[lo + i]]

    def velocity_unpack(self, sys, lo, count, ptr):
        v = self._view(ptr, count)
        for i in range(count):
            self.u[self.perm[lo + i]] = v[i]

    def step_finish(self):
        self.finished = self.u.copy()


def _split_worker(rank, world, port, q):
    import datetime

    import numpy as np
    import torch.distributed as dist
    from nuvort_b200.dist import TangleSplit
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    h = _FakeTangle(1001, seed=5)  # the same tangle on every rank
    TangleSplit(h, 0, dist, device="cpu").step()
    q.put((rank, bool(np.array_equal(h.finished[1:], h.truth[1:]))))
    dist.barrier()
    dist.destroy_process_group()


def _diverged_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    from nuvort_b200.dist import TangleSplit
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    h = _FakeTangle(1001 + rank, seed=5)  # the ranks' tangles differ: a diverged state
    try:
        TangleSplit(h, 0, dist, device="cpu").step()
        q.put((rank, "stepped"))
    except RuntimeError as e:
        q.put((rank, "refused" if "live counts differ" in str(e) else str(e)))
    dist.barrier()
    dist.destroy_process_group()


def test_tangle_split_refuses_diverged_ranks():
    # ranks whose live counts differ stop with an error on every rank, before the exchange
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_diverged_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert out == {0: "refused", 1: "refused"}


def test_tangle_split_over_two_gloo_ranks():
    # each rank computes half of the walk order; after the exchange both hold the full field
    from nuvort_b200.dist import split_ranges
    from nuvort_b200.dist import walk_range
    assert split_ranges(1001, 2) == [(1, 513), (513, 1002)]  # whole warps of 32 positions
    assert split_ranges(5, 3) == [(1, 1), (1, 1), (1, 6)]
    assert split_ranges(100, 8)[1] == (1, 33) and split_ranges(100, 8)[-1] == (97, 101)
    assert walk_range(513, 1002, 1064) == (513, 1065) and walk_range(1, 513, 1064) == (1, 513)
    assert walk_range(1, 1, 1064) == (1, 1)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
    assert out == {0: True, 1: True}
