"""GPU against the oracle at the sizes the benchmark runs, not only on small cases.

* The octree of the 1,048,576-point counterflow tangle (delta = 0.0005 cm, theta = 0.5):
  every node field bit for bit (src/tree.f90:38-157).
* The plain FP64 tree velocity of that tangle on a seeded 64-point subsample, against the
  oracle's calc_velocity at those points (src/timestep.f90:49-141, src/tree.f90:250-316),
  <= 1e-12 relative; the mixed-precision path on the same points within 1e-6 relative RMS.
* The FP64 direct-sum yardstick (nv_calc_velocity_direct_at), which every "error vs direct
  sum" figure is measured with, against the oracle's BS velocity at listed points
  (src/timestep.f90:74-98), <= 1e-12 relative, on a 32K and on the 1M tangle.
* 20 whole steps of a 32,768-point tree tangle at delta = 0.0005 cm: identical event logs,
  links and positions (within 1e-12 cm).  At this delta the next-but-one segment of a gently
  curved filament sits near the tree walk's absolute 4ac - b^2 < epsilon cut
  (src/tree.f90:303), so these steps exercise it.
"""
import numpy as np
import pytest

from helpers import rel_err, rms_rel, tangle
from nuvort_b200.abi import NV_VEL_BS, NV_VEL_TREE, make_params
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _config3_params(**over):
    kw = dict(dt=1e-6, delta=0.0005, box_size=0.1, velocity="Tree", tree_theta=0.5, corea=1.3e-8,
              alpha=(0.1, 0.01), normal_velocity="xflow", norm_vel_xflow=1.0)
    kw.update(over)
    return make_params(**kw)


@pytest.fixture(scope="module")
def tangle1m():
    return tangle(3, 0.0005, n_points=1048576)


def _subsample(n, k, seed):
    rng = np.random.Generator(np.random.PCG64(seed))
    return np.sort(rng.choice(np.arange(1, n + 1), size=k, replace=False)).astype(np.int32)


def test_tree_structure_1m_bit_exact(tangle1m):
    from nuvort_b200.api import Handle
    st = tangle1m
    p = _config3_params()
    with Handle(p, [st.pcount + 1024], states=[st]) as h:
        h.stage("ghostp")
        h.stage("construct_tree")
        tg = h.tree_dump()
    o = Oracle(p, st)
    o.stage("ghostp")
    o.stage("construct_tree")
    to = o.tree_dump()
    o.close()
    assert len(tg) == len(to) > 1_000_000
    for f in ("pos", "width", "cent", "circ", "pcount", "depth", "leaf", "first_next"):
        assert np.array_equal(tg[f], to[f]), f


def test_tree_velocity_1m_subsample(tangle1m):
    from nuvort_b200.api import Handle
    st = tangle1m
    sub = _subsample(st.pcount, 64, 2024)
    o = Oracle(_config3_params(), st)
    uo = o.calc_velocity_targets(NV_VEL_TREE, sub)
    o.close()
    with Handle(_config3_params(), [st.pcount + 1024], states=[st]) as h:
        ug = h.calc_velocity()[sub - 1]
    assert rel_err(ug, uo).max() <= 1e-12
    with Handle(_config3_params(precision=1), [st.pcount + 1024], states=[st]) as h:
        um = h.calc_velocity()[sub - 1]
    assert rms_rel(um, uo) <= 1e-6


@pytest.mark.parametrize("size,k", [(32768, 64), (1048576, 8)])
def test_direct_sum_yardstick_against_oracle(size, k, tangle1m):
    from nuvort_b200.api import Handle
    if size == 1048576:
        st, p = tangle1m, _config3_params()
    else:
        st = tangle(1, 0.001, n_points=size)
        p = make_params(dt=5e-6, delta=0.001, box_size=0.1, velocity="Tree", tree_theta=0.4, corea=1.3e-8,
                        alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.0, 0.0, 0.5))
    sub = _subsample(st.pcount, k, 77 + size)
    o = Oracle(p, st)
    uo = o.calc_velocity_targets(NV_VEL_BS, sub)
    o.close()
    with Handle(p, [st.pcount + 1024], states=[st]) as h:
        ud = h.calc_velocity_direct_at(0, sub)
    assert rel_err(ud, uo).max() <= 1e-12


def test_tree_tangle_small_delta_20_steps_events():
    from nuvort_b200.api import Handle
    st = tangle(5, 0.0005, n_points=32768)
    p = _config3_params()
    o = Oracle(p, st)
    o.step(20)
    with Handle(p, [st.pcount + 8192], states=[st]) as h:
        h.step(20)
        eg, a, cg = h.events(), h.download(), h.counters()
    eo, b, co = o.events(), o.download(), o.counters()
    o.close()
    assert len(eo) > 0
    assert eg == eo
    assert (cg.recon_count, cg.remove_count, cg.insert_count) == (co.recon_count, co.remove_count, co.insert_count)
    assert np.array_equal(a.infront, b.infront) and np.array_equal(a.behind, b.behind)
    assert np.max(np.abs(a.x - b.x)) < 1e-12
