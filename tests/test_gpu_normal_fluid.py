"""The normal-fluid fields of get_normal_velocity (src/normal_fluid.f90:83-118, 225-338) in the
mutual-friction term, GPU against the oracle: velocities within 1e-12 relative (the analytic
fields call the device sin/cos/cosh, within an ulp of the host's), and for the noisy flow
whole steps with identical events, the noise sample advancing once per step."""
import numpy as np
import pytest

from helpers import config0_params, rel_err, tangle
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _params(kind, **kw):
    return config0_params(alpha=(0.1, 0.01), normal_velocity=kind, norm_vel_xflow=0.7, **kw)


def _both(p, st, t=0.0, setup=None):
    from nuvort_b200.api import Handle
    with Handle(p, [st.pcount + 64], states=[st]) as h:
        h.set_clock(0, t, 3)
        if setup:
            setup(h, True)
        ug = h.calc_velocity()
    o = Oracle(p, st, t=t, itime=3)
    if setup:
        setup(o, False)
    return ug, o.calc_velocity()


@pytest.mark.parametrize("kind,extra", [("shear_xflow", dict(norm_shear_omega=2500.0)), ("ychannel", {}),
                                        ("channel", {})])
def test_analytic_fields(kind, extra):
    st = tangle(4, 0.002, n_rings=6)
    ug, uo = _both(_params(kind, **extra), st, t=3.7e-4)
    assert rel_err(ug, uo).max() <= TOL


def _grid(kind, seed=11):
    rng = np.random.default_rng(seed)
    if kind == "laizetDNS":
        nx, ny, nz = 128, 129, 84
        yp = -np.cos(np.linspace(0.0, np.pi, ny))  # a stretched wall-normal axis, ascending
    else:
        nx = ny = nz = 256
        yp = None
    u = rng.standard_normal((3, nz, ny, nx)) * 0.3
    return u, yp


@pytest.mark.parametrize("kind", ["laizetDNS", "turbDNS"])
def test_dns_grid_interpolation(kind):
    u, yp = _grid(kind)
    st = tangle(5, 0.002, n_rings=6)
    # the first ring moved across the lower x face: points below the first grid node of the
    # periodic x axis (turbDNS: x < -L/2), where the interpolation wraps to the last node
    n0 = next(k for k in range(1, st.pcount + 1) if st.infront[k - 1] < k)
    st.x[:n0, 0] += -0.052 - st.x[:n0, 0].min()
    def setup(obj, gpu):
        if gpu:
            obj.set_normal_fluid_grid(0, u, yp)
        else:
            obj.set_normal_fluid_grid(u, yp)
    ug, uo = _both(_params(kind), st, setup=setup)
    assert rel_err(ug, uo).max() <= TOL


def test_noisy_flow_whole_steps():
    from nuvort_b200.api import Handle
    noise = np.array([1.0, 0.3, -0.8, 2.1, 0.0, -1.5, 0.9])  # fewer samples than steps: wraps
    p = _params("noisey_xflow")
    st = tangle(6, 0.002, n_rings=8)
    o = Oracle(p, st)
    o.set_normal_fluid_noise(noise)
    with Handle(p, [st.pcount + 512], states=[st]) as h:
        h.set_normal_fluid_noise(0, noise)
        h.step(20)
        o.step(20)
        assert h.events() == o.events()
        a, b = h.download(), o.download()
    assert np.array_equal(a.infront, b.infront)
    assert np.max(np.abs(a.x - b.x)) < 1e-12


def test_missing_field_data_is_refused():
    from nuvort_b200.abi import NV_ERR_STATE
    from nuvort_b200.api import Handle, NuvortError
    st = tangle(6, 0.002, n_rings=3)
    for kind in ("noisey_xflow", "turbDNS"):
        with Handle(_params(kind), [st.pcount + 16], states=[st]) as h:
            with pytest.raises(NuvortError) as e:
                h.step(1)
            assert e.value.code == NV_ERR_STATE
