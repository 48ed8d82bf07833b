"""Shared builders for the parity tests: seeded tangles and matching parameter records."""
from __future__ import annotations

import numpy as np

from nuvort_b200.abi import make_params
from nuvort_b200.rings import random_rings, single_ring


def config0_params(**over):
    """Config 0: BS, brute pclose, no normal fluid, dt=2e-5 (periodic D=0.1, delta=0.002)."""
    kw = dict(dt=2e-5, delta=0.002, box_size=0.1, velocity="BS", corea=1.3e-8, tree_theta=0.0)
    kw.update(over)
    return make_params(**kw)


def config1_params(velocity="Tree", **over):
    """Config 1: theta=0.4, alpha=(0.1,0.01), v_n=(0,0,0.5), dt=5e-6, delta=0.001."""
    kw = dict(dt=5e-6, delta=0.001, box_size=0.1, velocity=velocity, corea=1.3e-8, tree_theta=0.4,
              alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.0, 0.0, 0.5))
    kw.update(over)
    return make_params(**kw)


def tangle(seed: int, delta: float, n_points=None, n_rings=None, box=0.1):
    return random_rings(seed, delta, (box, box, box), n_points=n_points, n_rings=n_rings)


def rel_err(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per-point relative error |a-b|/|b| (rows)."""
    nb = np.linalg.norm(b, axis=1)
    return np.linalg.norm(a - b, axis=1) / np.where(nb > 0, nb, 1.0)


def rms_rel(a: np.ndarray, b: np.ndarray) -> float:
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def small_rings(seed: int, n: int, npts: int, R: float, spread: float = 0.04):
    """n rings of npts points and radius R at random centres/orientations (no wrapping)."""
    from nuvort_b200.abi import State
    rng = np.random.default_rng(seed)
    xs, nx, pv, b = [], [], [], 0
    for _ in range(n):
        s = single_ring(R, npts, centre=rng.uniform(-spread, spread, 3), normal=rng.standard_normal(3))
        xs.append(s.x)
        nx.append(s.infront + b)
        pv.append(s.behind + b)
        b += npts
    x = np.ascontiguousarray(np.concatenate(xs))
    N = len(x)
    z = lambda: np.zeros((N, 3))
    return State(x=x, infront=np.concatenate(nx).astype(np.int32), behind=np.concatenate(pv).astype(np.int32),
                 u=z(), u1=z(), u2=z(), ghosti=z(), ghostb=z(), closest=np.zeros(N, np.int32),
                 closestd=np.zeros(N))
