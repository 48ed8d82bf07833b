"""Stage-by-stage parity of the GPU path against the oracle on identical inputs:
ghostp (bit-exact), pmotion (velocity + AB3 order ramp), enforce_boundary (bit-exact)."""
import numpy as np
import pytest

from helpers import config0_params, config1_params, rel_err, tangle
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _pair(p, st, cap=None):
    from nuvort_b200.api import Handle
    h = Handle(p, [cap or st.pcount + 256], states=[st])
    o = Oracle(p, st)
    return h, o


def test_ghostp_bit_exact():
    st = tangle(2, 0.002, n_rings=8)
    h, o = _pair(config0_params(), st)
    h.stage("ghostp")
    o.stage("ghostp")
    a, b = h.download(), o.download()
    assert np.array_equal(a.ghosti, b.ghosti) and np.array_equal(a.ghostb, b.ghostb)
    h.close()


def test_pmotion_three_steps_order_ramp():
    # Euler, then AB2, then AB3 (timestep.f90:31-39) on three successive pmotion calls.
    st = tangle(4, 0.002, n_rings=6)
    p = config0_params()
    h, o = _pair(p, st)
    for _ in range(3):
        for s in ("ghostp", "pmotion"):
            h.stage(s)
            o.stage(s)
        a, b = h.download(), o.download()
        assert np.max(np.abs(a.x - b.x)) <= 1e-15
        assert rel_err(a.u1, b.u1).max() <= 1e-12
    h.close()


def test_enforce_boundary_bit_exact():
    st = tangle(6, 0.002, n_rings=8)
    st.x[::7] += 0.051  # push some points outside the box
    h, o = _pair(config0_params(), st)
    h.stage("enforce_boundary")
    o.stage("enforce_boundary")
    assert np.array_equal(h.download().x, o.download().x)
    h.close()


def test_upload_download_round_trip_and_checks():
    # every array of the host state goes up and comes back unchanged (links 1-based within
    # the system, the slots past pcount empty); bad links are refused
    from nuvort_b200.api import Handle, NuvortError
    from nuvort_b200.abi import State
    st = tangle(2, 0.002, n_rings=5)
    n = st.pcount
    rng = np.random.default_rng(7)
    full = State(x=st.x.copy(), infront=st.infront.copy(), behind=st.behind.copy(),
                 u=rng.standard_normal((n, 3)), u1=rng.standard_normal((n, 3)), u2=rng.standard_normal((n, 3)),
                 ghosti=rng.standard_normal((n, 3)), ghostb=rng.standard_normal((n, 3)),
                 closest=rng.integers(0, n + 1, n).astype(np.int32), closestd=rng.standard_normal(n))
    with Handle([config0_params()] * 2, [n + 100, n + 50], states=[st, st]) as h:
        h.upload(1, full)
        back = h.download(1)
        for name in ("x", "u", "u1", "u2", "ghosti", "ghostb", "closestd", "infront", "behind", "closest"):
            assert np.array_equal(getattr(back, name), getattr(full, name)), name
        assert h.counters(1).live == int(np.count_nonzero(st.infront))
        assert np.array_equal(h.download(0).x, st.x)  # the other system untouched
        part = h.download(1, out=State.empty(n + 50), fields=("x", "infront"))
        assert part.u is None and np.array_equal(part.x, full.x) and np.array_equal(part.infront, full.infront)
        # a refused upload leaves the system exactly as it was
        moved = State(x=st.x + 0.001, infront=st.infront.copy(), behind=st.behind.copy())
        bad = State(x=moved.x, infront=st.infront.copy(), behind=st.behind.copy())
        bad.infront[3] = n + 1
        with pytest.raises(NuvortError, match="out of range"):
            h.upload(1, bad)
        bad = State(x=moved.x, infront=st.infront.copy(), behind=st.behind.copy())
        bad.behind[5] = 0
        with pytest.raises(NuvortError, match="disagree"):
            h.upload(1, bad)
        bad = State(x=moved.x, infront=st.infront.copy(), behind=st.behind.copy(),
                    closest=np.full(n, -1, np.int32))
        with pytest.raises(NuvortError, match="out of range"):
            h.upload(1, bad)
        back = h.download(1)
        for name in ("x", "u", "u1", "u2", "ghosti", "ghostb", "closestd", "infront", "behind", "closest"):
            assert np.array_equal(getattr(back, name), getattr(full, name)), name
        assert h.counters(1).live == int(np.count_nonzero(st.infront)) and h.counters(1).pcount == n
