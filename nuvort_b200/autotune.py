"""Autotuner: the direct-sum / tree crossover of the batched ensemble, and the block shapes of
the velocity pass (tune_launch_shapes), measured on the device.

A system of N points costs the direct sum 27 N^2 pair terms and the tree walk roughly
27 N log N node visits plus a tree build, so below some N the direct sum is cheaper.  The
crossover depends on the GPU, the precision and the tree's opening angle; it is measured here
rather than assumed.  For each trial size N, a handle holding enough systems of N points to
fill the GPU (as they are in a batch) runs a few whole steps with the direct sum and with the
tree walk; the device time of the velocity stage plus, for the tree, the tree build, per
point, is compared.  The crossover is the smallest trial size at which the tree is faster
(interpolated between the two bracketing sizes), or the largest tried size if the direct sum
always wins.

The result is cached per (device name, precision, delta, theta) in a JSON file beside this
module so that later runs skip the measurement.
"""
from __future__ import annotations

import json
import os
from typing import Dict, Sequence

from . import api
from .abi import make_params
from .rings import random_rings

_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "autotune.json")


def _stage_cost(params, states, steps: int, tree: bool) -> float:
    """Device ms per point per step of the velocity stage (and the tree build if tree)."""
    caps = [int(s.pcount * 1.6) + 256 for s in states]
    h = api.Handle(params, caps, states=states)
    try:
        h.step(1)  # warm-up: graph capture, first tree build
        t0 = h.stage_times()
        h.step(steps)
        t1 = h.stage_times()
        ms = t1["velocity"] - t0["velocity"]
        if tree:
            ms += t1["tree"] - t0["tree"]
        pts = sum(s.pcount for s in states) * steps
        return ms / pts
    finally:
        h.close()


def tune_crossover(device: int = 0, precision: str = "mixed", delta: float = 0.002, theta: float = 0.4,
                   sizes: Sequence[int] = (500, 1000, 1500, 2000, 3000, 4000, 6000, 8000),
                   batch_points: int = 1 << 17, steps: int = 2, use_cache: bool = True) -> Dict:
    """Measure the direct/tree crossover (points per system) on this GPU; see the module doc.
    use_cache=False neither reads nor writes the cache."""
    import torch

    name = torch.cuda.get_device_name(device)
    key = f"{name}|{precision}|{delta:g}|{theta:g}"
    if use_cache and os.path.exists(_CACHE):
        try:
            with open(_CACHE) as f:
                cached = json.load(f).get(key)
            if cached:
                return dict(cached, cached=True)
        except (OSError, ValueError):
            pass
    trials = []
    for n in sizes:
        nsys = max(1, batch_points // n)
        states = [random_rings(7919 + 31 * k, delta, (0.1, 0.1, 0.1), n_points=n) for k in range(nsys)]
        common = dict(dt=2e-5, delta=delta, box_size=0.1, corea=1.3e-8, tree_theta=theta, alpha=(0.1, 0.01),
                      normal_velocity="uniform", norm_vel_vec=(0.0, 0.0, 0.5), precision=precision)
        direct = _stage_cost([make_params(velocity="BS", **common)] * nsys, states, steps, tree=False)
        tree = _stage_cost([make_params(velocity="Tree", **common)] * nsys, states, steps, tree=True)
        trials.append({"points": n, "systems": nsys, "direct_ms_per_point": direct, "tree_ms_per_point": tree})
    crossover = sizes[-1]
    for a, b in zip(trials, trials[1:]):
        da = a["tree_ms_per_point"] - a["direct_ms_per_point"]
        db = b["tree_ms_per_point"] - b["direct_ms_per_point"]
        if da > 0 >= db:  # the tree becomes the cheaper one between a and b
            f = da / (da - db)
            crossover = int(round(a["points"] + f * (b["points"] - a["points"])))
            break
    else:
        if trials and trials[0]["tree_ms_per_point"] <= trials[0]["direct_ms_per_point"]:
            crossover = sizes[0]
    result = {"crossover": crossover, "device": name, "precision": precision, "delta": delta, "theta": theta,
              "trials": trials}
    if not use_cache:
        return dict(result, cached=False)
    os.makedirs(os.path.dirname(_CACHE), exist_ok=True)
    try:
        with open(_CACHE) as f:
            allc = json.load(f)
    except (OSError, ValueError):
        allc = {}
    allc[key] = result
    with open(_CACHE, "w") as f:
        json.dump(allc, f, indent=1)
    return dict(result, cached=False)


def _velocity_ms(handle, repeats: int) -> float:
    """Host-timed velocity pass of every system of `handle` (nv_calc_velocity, which waits for
    its stream): the fastest of `repeats` after one warm-up."""
    import time
    handle.calc_velocity(0)
    best = float("inf")
    for _ in range(repeats):
        t0 = time.perf_counter()
        handle.calc_velocity(0)
        best = min(best, (time.perf_counter() - t0) * 1e3)
    return best


def tune_launch_shapes(handle, repeats: int = 3) -> Dict:
    """Block shapes of the velocity pass, measured on `handle`'s own systems, the fastest kept
    (set on the handle):

    * walk_parts (nv_set_walk_parts) for tree-walk systems: the mixed walk's central image over
      1, 2, 4 or 8 groups of root children (more, shorter blocks for small systems); the
      plain FP64 walk's unshifted and shifted images on one or two threads per target;
    * direct split (nv_set_direct_split) for plain FP64 direct-sum systems: one thread per
      target (64) or 8, 4, 2, 1 targets per block, each target's terms spread over the block.

    The plain FP64 choices do not change a result (both walk splits and every direct split add
    the same terms in the reference's order); the mixed walk's parts group its FP32 partial
    sums differently (within the mixed tolerance).  Runs velocity passes only: the systems'
    positions and links are unchanged (the next step recomputes the velocities)."""
    from .abi import NV_PREC_MIXED, NV_VEL_BS, NV_VEL_TREE
    mixed = any(p.precision == NV_PREC_MIXED for p in handle.params)
    tree = any(p.velocity == NV_VEL_TREE for p in handle.params)
    direct = not mixed and any(p.velocity == NV_VEL_BS for p in handle.params)
    def trial(setter, candidates):
        ms = {}
        for c in candidates:
            setter(c)
            ms[c] = _velocity_ms(handle, repeats)
        choice = min(ms, key=ms.get)
        setter(choice)
        return {"choice": choice, "ms": ms}

    out: Dict = {}
    if tree:
        out["walk_parts"] = trial(handle.set_walk_parts, (1, 2, 4, 8) if mixed else (1, 2))
    if direct:
        out["direct_split"] = trial(handle.set_direct_split, (64, 8, 4, 2, 1))
    return out
