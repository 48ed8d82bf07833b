"""CPU checks of the oracle (the line-by-line C++ restatement of the reference Fortran).

The reference ships no tests or golden vectors, so the oracle is checked against the one
analytic answer the reference itself prints (the ring self-velocity of
src/initial_cond.f90:16), against the limits the algorithms must reach (tree -> direct sum
as theta -> 0), against topology invariants, and against the committed fixtures in
tests/golden (which pin its own outputs so that later changes cannot drift silently).
"""
import math
import os

import numpy as np
import pytest

from helpers import config0_params, config1_params, rel_err, rms_rel, tangle
from nuvort_b200.abi import NV_VEL_BS, NV_VEL_LIA, NV_VEL_TREE, make_params
from nuvort_b200.rings import single_ring
import oracle
from oracle import Oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_ring_self_velocity_known_answer():
    # src/initial_cond.f90:16: v = Gamma/(4 pi R) (ln(8R/a0) - 1/2)
    R, n, a0, gamma = 0.02, 126, 1.3e-8, 9.97e-4
    st = single_ring(R, n)
    p = make_params(dt=1e-5, delta=0.002, box_size=1.0, velocity="BS", corea=a0)
    u = Oracle(p, st).calc_velocity()
    v = gamma / (4 * math.pi * R) * (math.log(8 * R / a0) - 0.5)
    assert abs(u[:, 2].mean() / v - 1) < 5e-3
    # the ring translates rigidly: transverse components vanish on average
    assert abs(u[:, 0].mean()) < 1e-6 and abs(u[:, 1].mean()) < 1e-6


def test_tree_converges_to_direct_sum():
    st = tangle(11, 0.001, n_points=2048)
    errs = []
    for theta in (0.4, 0.1, 0.002):
        o = Oracle(config1_params("Tree", tree_theta=theta), st)
        tg = np.arange(1, st.pcount + 1)
        ut = o.calc_velocity_targets(NV_VEL_TREE, tg)
        ub = o.calc_velocity_targets(NV_VEL_BS, tg)
        errs.append(rms_rel(ut, ub))
    assert errs[0] > errs[1] > errs[2]
    assert errs[2] < 1e-3


def test_oracle_thread_count_does_not_change_results():
    st = tangle(3, 0.002, n_rings=4)
    res = []
    for nt in (1, 4):
        oracle.set_threads(nt)
        o = Oracle(config0_params(), st)
        o.step(10)
        res.append(o.download())
    oracle.set_threads(os.cpu_count() or 1)
    assert np.array_equal(res[0].x, res[1].x)
    assert np.array_equal(res[0].infront, res[1].infront)


def _check_links(st):
    live = np.nonzero(st.infront)[0] + 1
    nxt, prv = st.infront, st.behind
    for k in live:
        assert prv[nxt[k - 1] - 1] == k
        assert nxt[prv[k - 1] - 1] == k
    # every loop has at least 4 points (loop_killer, src/reconnection.f90:155-182)
    seen = set()
    for k in live:
        if k in seen:
            continue
        n, j = 0, k
        while True:
            seen.add(j)
            n += 1
            j = nxt[j - 1]
            if j == k:
                break
        assert n >= 4


def test_topology_invariants_config0():
    st = tangle(0, 0.002, n_rings=8)
    o = Oracle(config0_params(), st)
    o.step(60)
    out = o.download()
    _check_links(out)
    c = o.counters()
    assert c.insert_count > 0
    assert c.live == int(np.count_nonzero(out.infront))


def test_timestep_check_matches_reference_bound():
    # dt_max for delta = 0.002, 0.001, 0.0005 (src/initial.f90:169-180)
    for delta, dtmax in ((0.002, 9.9e-5), (0.001, 2.7e-5), (0.0005, 7.2e-6)):
        dm = delta / 2
        val = abs(dm ** 2 / (9.97e-4 * math.log(dm / (math.pi * 1.3e-8))))
        assert abs(val / dtmax - 1) < 0.05


@pytest.mark.parametrize("name", ["config0_bs", "config1_tree_small"])
def test_golden_fixture(name):
    path = os.path.join(GOLDEN, name + ".npz")
    g = np.load(path)
    from golden.make_golden import CASES
    st, p, kind = CASES[name]()
    o = Oracle(p, st)
    if kind == "velocity":
        u = o.calc_velocity()
        assert np.array_equal(u, g["u"]), "oracle velocity drifted from its fixture"
    if "x_after" in g:
        o2 = Oracle(p, st)
        o2.step(int(g["nsteps"]))
        out = o2.download()
        assert np.array_equal(out.x, g["x_after"])
        assert np.array_equal(out.infront, g["infront_after"])
        ev = np.array(o2.events(), dtype=np.int32).reshape(-1, 4)
        assert np.array_equal(ev, g["events"])
    if "tree_cent" in g:
        o.stage("ghostp")
        o.stage("construct_tree")
        tr = o.tree_dump()
        assert np.array_equal(tr["cent"], g["tree_cent"])
        assert np.array_equal(tr["pcount"], g["tree_pcount"])
