"""Autotuner for the batched ensemble: the direct-sum / tree crossover, measured on the device.

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
