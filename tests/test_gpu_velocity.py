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
