"""Batched ensembles: several independent systems of uneven size in one handle, with their
own parameters.  Each system must evolve exactly as it does alone (plain path: bit for bit;
mixed path: within 1e-6 relative RMS)."""
import numpy as np
import pytest

from helpers import config0_params, config1_params, rel_err, rms_rel, tangle
from nuvort_b200.abi import make_params
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _ensemble():
    states = [tangle(40, 0.002, n_rings=3), tangle(41, 0.002, n_points=1500), tangle(42, 0.002, n_rings=6),
              tangle(43, 0.002, n_points=700)]
    params = [config0_params(alpha=(0.05, 0.01), normal_velocity="uniform", norm_vel_vec=(0.3, 0.0, 0.1)),
              config0_params(velocity="Tree", tree_theta=0.4, alpha=(0.2, 0.0), normal_velocity="uniform",
                             norm_vel_vec=(0.0, 0.8, 0.0)),
              config0_params(),
              config0_params(velocity="Tree", tree_theta=0.4, alpha=(0.1, 0.02), normal_velocity="xflow",
                             norm_vel_xflow=0.6)]
    return states, params


def test_batched_plain_equals_systems_alone():
    from nuvort_b200.api import Handle
    states, params = _ensemble()
    caps = [s.pcount + 600 for s in states]
    h = Handle(params, caps, states=states)
    h.step(30)
    for k, (st, p) in enumerate(zip(states, params)):
        o = Oracle(p, st)
        o.step(30)
        a, b = h.download(k), o.download()
        assert h.events(k) == o.events(), k
        assert np.array_equal(a.infront, b.infront), k
        assert np.max(np.abs(a.x - b.x)) < 1e-12, k
    h.close()


def test_batched_velocity_mixed():
    from nuvort_b200.api import Handle
    states, params = _ensemble()
    pm = []
    for p in params:
        q = type(p).from_buffer_copy(p)
        q.precision = 1
        pm.append(q)
    caps = [s.pcount + 600 for s in states]
    hp = Handle(params, caps, states=states)
    hm = Handle(pm, caps, states=states)
    for k in range(len(states)):
        up, um = hp.calc_velocity(k), hm.calc_velocity(k)
        assert rms_rel(um, up) <= 1e-6, k
    hp.close()
    hm.close()


def test_autotuned_crossover_is_measured():
    # two small trial sizes: the tuner runs both methods on batches of systems and returns a
    # crossover inside the tried range, with the per-point costs it measured
    from nuvort_b200.autotune import tune_crossover
    r = tune_crossover(sizes=(400, 1600), batch_points=1 << 13, steps=1, use_cache=False)
    assert 400 <= r["crossover"] <= 1600
    assert len(r["trials"]) == 2
    for t in r["trials"]:
        assert t["direct_ms_per_point"] > 0 and t["tree_ms_per_point"] > 0


def _velocities(h, n):
    return np.concatenate([h.calc_velocity(s) for s in range(n)])


def test_launch_shapes_tuned_on_the_handle():
    # the ensemble's direct-sum and tree systems: the tuner times each candidate shape, keeps
    # the fastest, and the plain FP64 velocities are bit-identical under the chosen shapes;
    # the mixed walk's parts regroup FP32 partial sums only (within 1e-7 relative RMS)
    from nuvort_b200.api import Handle
    from nuvort_b200.autotune import tune_launch_shapes
    states, params = _ensemble()
    caps = [s.pcount + 600 for s in states]
    with Handle(params, caps, states=states) as h:
        before = _velocities(h, len(states))
        r = tune_launch_shapes(h, repeats=1)
        assert r["walk_parts"]["choice"] in (1, 2) and set(r["walk_parts"]["ms"]) == {1, 2}
        assert r["direct_split"]["choice"] in (64, 8, 4, 2, 1) and len(r["direct_split"]["ms"]) == 5
        assert all(v > 0 for v in r["direct_split"]["ms"].values())
        assert np.array_equal(_velocities(h, len(states)), before)
    mixed = []
    for p in params:
        q = type(p).from_buffer_copy(p)
        q.precision = 1
        mixed.append(q)
    with Handle(mixed, caps, states=states) as h:
        before = _velocities(h, len(states))
        r = tune_launch_shapes(h, repeats=1)
        assert r["walk_parts"]["choice"] in (1, 2, 4, 8) and "direct_split" not in r
        assert rms_rel(_velocities(h, len(states)), before) <= 1e-7
