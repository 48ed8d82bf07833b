"""Seeded synthetic filament tangles: random vortex rings in a periodic box.

These stand in for the reference's initial conditions (setup_random_loops,
src/initial_cond.f90:115-191, draws equal loops by Euler-angle rotation); the workloads
here need rings of random radius and orientation and an exact point count:

* centre uniform in the box, unit normal uniform on the sphere (normalised Gaussian
  triple), radius uniform in [rmin, rmax];
* n = ceil(2*pi*R/delta) points per ring, so every chord is below delta and no point is
  inserted at the first step;
* points wrapped into [-L/2, L/2) on every axis; slots numbered ring after ring, each
  point's ``infront`` the next point of its ring (wrapping inside the ring), ``behind`` the
  previous, as in the reference's loop set-ups;
* for an exact total N: whole rings are added while the next one fits; the remainder m
  becomes a last ring of radius 0.999*m*delta/(2*pi), or, when m < 32, extra points on the
  previous ring.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .abi import State


def _ring_points(c: np.ndarray, nrm: np.ndarray, R: float, n: int) -> np.ndarray:
    a = np.array([1.0, 0.0, 0.0]) if abs(nrm[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(nrm, a)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(nrm, e1)
    phi = 2.0 * np.pi * np.arange(n) / n
    return c[None, :] + R * (np.cos(phi)[:, None] * e1[None, :] + np.sin(phi)[:, None] * e2[None, :])


def ring_specs(seed: int, delta: float, box: Sequence[float] = (0.1, 0.1, 0.1),
               n_rings: Optional[int] = None, n_points: Optional[int] = None,
               rmin: float = 0.015, rmax: float = 0.03) -> List[Tuple[np.ndarray, np.ndarray, float, int]]:
    """Draw (centre, normal, radius, points) for each ring."""
    if (n_rings is None) == (n_points is None):
        raise ValueError("give exactly one of n_rings, n_points")
    rng = np.random.Generator(np.random.PCG64(seed))
    L = np.asarray(box, dtype=np.float64)
    specs: List[Tuple[np.ndarray, np.ndarray, float, int]] = []
    total = 0
    while True:
        c = rng.uniform(-0.5, 0.5, size=3) * L
        nrm = rng.standard_normal(3)
        nrm /= np.linalg.norm(nrm)
        R = float(rng.uniform(rmin, rmax))
        n = int(math.ceil(2.0 * math.pi * R / delta))
        if n_rings is not None:
            specs.append((c, nrm, R, n))
            if len(specs) == n_rings:
                return specs
            continue
        if total + n <= n_points:
            specs.append((c, nrm, R, n))
            total += n
            if total == n_points:
                return specs
            continue
        m = n_points - total
        if m >= 32 or not specs:
            specs.append((c, nrm, 0.999 * m * delta / (2.0 * math.pi), m))
        else:
            pc, pn, pR, pnum = specs[-1]
            specs[-1] = (pc, pn, pR, pnum + m)
        return specs


def random_rings(seed: int, delta: float, box: Sequence[float] = (0.1, 0.1, 0.1),
                 n_rings: Optional[int] = None, n_points: Optional[int] = None,
                 rmin: float = 0.015, rmax: float = 0.03) -> State:
    """A State holding the seeded ring tangle (u, u1, u2 zero; ghosts unset)."""
    L = np.asarray(box, dtype=np.float64)
    specs = ring_specs(seed, delta, box, n_rings=n_rings, n_points=n_points, rmin=rmin, rmax=rmax)
    xs, nxt, prv = [], [], []
    base = 0
    for c, nrm, R, n in specs:
        xs.append(_ring_points(c, nrm, R, n))
        k = np.arange(n)
        nxt.append(base + 1 + (k + 1) % n)
        prv.append(base + 1 + (k - 1) % n)
        base += n
    x = np.concatenate(xs)
    x = x - L[None, :] * np.floor((x + 0.5 * L[None, :]) / L[None, :])
    x = np.where(x >= 0.5 * L[None, :], x - L[None, :], x)
    npts = x.shape[0]
    z = lambda: np.zeros((npts, 3), np.float64)
    return State(x=np.ascontiguousarray(x), infront=np.concatenate(nxt).astype(np.int32),
                 behind=np.concatenate(prv).astype(np.int32), u=z(), u1=z(), u2=z(),
                 ghosti=z(), ghostb=z(), closest=np.zeros(npts, np.int32),
                 closestd=np.zeros(npts, np.float64))


def single_ring(R: float, n: int, centre=(0.0, 0.0, 0.0), normal=(0.0, 0.0, 1.0)) -> State:
    """One ring of n points (the single_loop set-up of src/initial_cond.f90:9-35, any axis)."""
    nrm = np.asarray(normal, np.float64)
    nrm /= np.linalg.norm(nrm)
    x = _ring_points(np.asarray(centre, np.float64), nrm, R, n)
    k = np.arange(n)
    z = lambda: np.zeros((n, 3), np.float64)
    return State(x=np.ascontiguousarray(x), infront=(1 + (k + 1) % n).astype(np.int32),
                 behind=(1 + (k - 1) % n).astype(np.int32), u=z(), u1=z(), u2=z(), ghosti=z(),
                 ghostb=z(), closest=np.zeros(n, np.int32), closestd=np.zeros(n, np.float64))


def ensemble(seed: int, n_systems: int, nmin: int, nmax: int, delta: float,
             box: Sequence[float] = (0.1, 0.1, 0.1), log_uniform: bool = True) -> List[State]:
    """Independent ring tangles with point counts drawn log-uniformly (or uniformly)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    if log_uniform:
        counts = np.exp(rng.uniform(math.log(nmin), math.log(nmax), size=n_systems))
    else:
        counts = rng.uniform(nmin, nmax, size=n_systems)
    counts = np.maximum(np.round(counts).astype(int), 64)
    sub = rng.integers(0, 2**31 - 1, size=n_systems)
    return [random_rings(int(s), delta, box, n_points=int(n)) for s, n in zip(sub, counts)]


def _pinned_state(x: np.ndarray, infront: np.ndarray, behind: np.ndarray, wpinned: np.ndarray,
                  pinnedi: np.ndarray, pinnedb: np.ndarray) -> State:
    n = x.shape[0]
    z = lambda: np.zeros((n, 3), np.float64)
    return State(x=np.ascontiguousarray(x), infront=infront.astype(np.int32), behind=behind.astype(np.int32),
                 u=z(), u1=z(), u2=z(), ghosti=z(), ghostb=z(), closest=np.zeros(n, np.int32),
                 closestd=np.zeros(n, np.float64), wpinned=wpinned.astype(np.int32),
                 pinnedi=pinnedi.astype(np.int32), pinnedb=pinnedb.astype(np.int32))


def half_loop(n: int, delta: float, box: Sequence[float] = (0.1, 0.1, 0.1), axis: int = 0) -> State:
    """A half ring of n points standing on the solid wall at +L/2 of ``axis`` (0: x, the
    setup_half_loop of src/initial_cond.f90:41-75; 2: z, setup_half_loopz :79-113): radius
    0.75 n delta / pi, its first point pinned behind and its last pinned in front, both to
    that wall.  Only x (in the x-y plane) and z (in the z-y plane) are set up there."""
    if axis not in (0, 2):
        raise ValueError("half loops stand on the x or z wall")
    R = (0.75 * n * delta) / math.pi
    k = np.arange(n)
    s = np.sin(math.pi * k / (n - 1))
    c = np.cos(math.pi * k / (n - 1))
    x = np.zeros((n, 3), np.float64)
    x[:, axis] = 0.5 * box[axis] - R * s
    x[:, 1] = R * c
    infront = np.minimum(k + 2, n)  # 1-based: the last point is its own infront
    behind = np.maximum(k, 1)       # the first point is its own behind
    w = np.zeros((n, 3), np.int32)
    w[0, axis] = w[-1, axis] = 1
    pi_ = np.zeros(n, np.int32)
    pb_ = np.zeros(n, np.int32)
    pi_[-1] = 1
    pb_[0] = 1
    return _pinned_state(x, infront, behind, w, pi_, pb_)


def lattice(line_count: int, delta: float, box: Sequence[float] = (0.1, 0.1, 0.1),
            lattice_ratio: float = 0.5) -> State:
    """Straight lines from the +z wall to the -z wall on a triangular (hexagonal-number)
    lattice, as setup_lattice (src/initial_cond.f90:252-318) draws them:
    3 line_count (line_count - 1) + 1 lines of nint(L_z / (0.75 delta)) points each; a line's
    first point sits on the +z wall pinned behind (wpinned 0,0,1), its last on the -z wall
    pinned in front (wpinned 0,0,-1)."""
    nl = 3 * line_count * (line_count - 1) + 1
    per = int(math.floor(box[2] / (0.75 * delta) + 0.5))  # nint
    r = [0.0]
    th = [0.0]
    for i in range(2, line_count + 1):
        for j in range(1, (i - 1) * 6 + 1):
            t = 2.0 * math.pi * (j - 1) / ((i - 1) * 6)
            th.append(t)
            r.append(0.5 * lattice_ratio * min(box[0], box[1]) * ((i - 1) / (line_count - 1)) *
                     math.cos(math.pi / 6) / math.cos(math.fmod(t, 2 * math.pi / 6) - math.pi / 6))
    n = nl * per
    x = np.zeros((n, 3), np.float64)
    infront = np.zeros(n, np.int64)
    behind = np.zeros(n, np.int64)
    w = np.zeros((n, 3), np.int32)
    pi_ = np.zeros(n, np.int32)
    pb_ = np.zeros(n, np.int32)
    j = np.arange(per)
    for i in range(nl):
        rows = i * per + j  # 0-based rows; slot = row + 1
        x[rows, 0] = r[i] * math.cos(th[i])
        x[rows, 1] = r[i] * math.sin(th[i])
        x[rows, 2] = box[2] / 2.0 - box[2] * j / (per - 1)
        infront[rows] = rows + 2
        behind[rows] = rows
        infront[rows[-1]] = rows[-1] + 1
        behind[rows[0]] = rows[0] + 1
        pb_[rows[0]] = 1
        w[rows[0], 2] = 1
        pi_[rows[-1]] = 1
        w[rows[-1], 2] = -1
    return _pinned_state(x, infront, behind, w, pi_, pb_)
