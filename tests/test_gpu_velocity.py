"""calc_velocity on the GPU against the CPU oracle (plain FP64 path).

The plain path keeps the reference's operation order with one rounding per operation, so
velocities agree bit for bit apart from the device log() in the local term (<= 1 ulp of
beta).  Tolerance: 1e-12 relative per point, as the plain path promises."""
import numpy as np
import pytest

from helpers import config0_params, config1_params, rel_err, tangle
from nuvort_b200.abi import make_params
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _gpu_velocity(p, st, cap=None):
    from nuvort_b200.api import Handle
    with Handle(p, [cap or st.pcount + 64], states=[st]) as h:
        return h.calc_velocity()


@pytest.mark.parametrize("velocity", ["BS", "LIA"])
def test_velocity_config0(velocity):
    st = tangle(0, 0.002, n_rings=8)
    p = config0_params(velocity=velocity)
    ug = _gpu_velocity(p, st)
    uo = Oracle(p, st).calc_velocity()
    e = rel_err(ug, uo)
    assert e.max() <= TOL, e.max()
    # most points agree bit for bit
    assert np.mean(np.all(ug == uo, axis=1)) > 0.3


def test_velocity_bs_mutual_friction_open_box():
    st = tangle(5, 0.002, n_rings=6)
    p = make_params(dt=2e-5, delta=0.002, box_size=0.1, velocity="BS", corea=1.3e-8,
                    alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.2, -0.1, 0.5),
                    super_velocity=(0.01, 0.0, -0.02), boundary_y="open")
    ug = _gpu_velocity(p, st)
    uo = Oracle(p, st).calc_velocity()
    assert rel_err(ug, uo).max() <= TOL


def test_velocity_bs_with_empty_slots():
    st = tangle(7, 0.002, n_rings=5)
    # clear one whole ring (slots of the first ring) to make holes
    first = st.infront[0]
    n0 = 0
    k = 1
    while True:
        n0 += 1
        k = st.infront[k - 1]
        if k == 1:
            break
    st.infront[:n0] = 0
    st.behind[:n0] = 0
    st.x[:n0] = 0
    p = config0_params()
    ug = _gpu_velocity(p, st, cap=st.pcount + 10)
    uo = Oracle(p, st).calc_velocity()
    assert np.all(ug[:n0] == 0)
    assert rel_err(ug[n0:], uo[n0:]).max() <= TOL


def test_velocity_bs_4096():
    st = tangle(1, 0.001, n_points=4096)
    p = config1_params("BS")
    ug = _gpu_velocity(p, st)
    uo = Oracle(p, st).calc_velocity()
    assert rel_err(ug, uo).max() <= TOL


def test_direct_split_bit_identical_to_one_thread_per_target():
    # the split kernel computes the terms of each target's sum on many threads and adds them
    # in the reference's order on one lane per component: the same bits as one thread per
    # target, for every split, with holes (empty slots) and mutual friction
    from nuvort_b200.api import Handle
    st = tangle(11, 0.002, n_rings=9)
    # empty the third ring (its slots run from the slot after the second ring's last one)
    ends = [k for k in range(1, st.pcount + 1) if st.infront[k - 1] < k]  # last slot of each ring
    a, b = ends[1], ends[2]  # 0-based slice [a, b) = 1-based slots a+1..b
    st.infront[a:b] = 0
    st.behind[a:b] = 0
    st.x[a:b] = 0
    p = config0_params(alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.1, 0.0, 0.3))
    uo = Oracle(p, st).calc_velocity()
    live = st.infront > 0
    res = {}
    with Handle(p, [st.pcount + 77], states=[st]) as h:
        for g in (64, 1, 2, 4, 8, 0):
            h.set_direct_split(g)
            res[g] = h.calc_velocity()
    for g, u in res.items():
        assert np.array_equal(u, res[64]), g
    assert np.all(res[64][~live] == 0)
    assert rel_err(res[64][live], uo[live]).max() <= TOL


@pytest.mark.parametrize("split", [64, 4, 0])
def test_direct_at_listed_targets_split(split):
    # the FP64 direct-sum yardstick at listed slots, in list order (repeats and unsorted)
    from nuvort_b200.abi import NV_VEL_BS
    from nuvort_b200.api import Handle
    st = tangle(1, 0.001, n_points=4096)
    p = config1_params("Tree")
    tg = np.array([4096, 1, 17, 17, 2048, 3000, 5, 999], np.int32)
    uo = Oracle(p, st).calc_velocity_targets(NV_VEL_BS, tg)
    with Handle(p, [st.pcount + 64], states=[st]) as h:
        h.set_direct_split(split)
        ud = h.calc_velocity_direct_at(0, tg)
    assert rel_err(ud, uo).max() <= TOL
