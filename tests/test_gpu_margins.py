"""Event margins (nv_set_event_margins / nv_event_margins_get): how close the topology tests
came to deciding the other way.  The plain path against the oracle's record of the same
tests: pinsert's margin equal (the same lengths), the others never above the oracle's (the
device evaluates every value the reference does, and some stale ones more); then the mixed
path's margins against the largest position difference it makes to the plain path."""
import numpy as np
import pytest

from helpers import config0_params, config1_params, tangle
from oracle import Oracle

pytestmark = pytest.mark.gpu

KEYS = ("insert", "remove", "recon_distance", "recon_dot")


def _run(p, st, steps, extra=8192):
    from nuvort_b200.api import Handle
    h = Handle(p, [st.pcount + extra], states=[st])
    h.set_event_margins(True)
    h.step(steps)
    return h


@pytest.mark.parametrize("which", ["bs", "tree"])
def test_margins_against_oracle(which):
    if which == "bs":
        p, st, steps = config0_params(), tangle(0, 0.002, n_rings=8), 60
    else:
        p, st, steps = config1_params("Tree"), tangle(1, 0.001, n_points=4096), 20
    h = _run(p, st, steps)
    mg = h.event_margins()
    ev = h.events()
    h.close()
    o = Oracle(p, st)
    o.set_event_margins(True)
    o.step(steps)
    mo = o.event_margins()
    assert ev == o.events()
    assert mg["insert"] == mo["insert"]
    for k in KEYS[1:]:
        assert 0.0 <= mg[k] <= mo[k], (k, mg[k], mo[k])
    assert all(v < 1e300 for v in mo.values())  # every test ran


def test_mixed_margins_recorded_beside_equal_events():
    # The mixed path's positions differ from the plain path's by ~1e-11 cm here, while some
    # pinsert test comes within ~1e-9 delta of its threshold: the margins do not bound the
    # event equality (which holds for this seeded case); they say how close it came.
    p = config1_params("Tree")
    st = tangle(2, 0.001, n_points=16384)
    hp = _run(p, st, 20)
    pm = config1_params("Tree", precision="mixed")
    hm = _run(pm, st, 20)
    assert hm.events() == hp.events()
    a, b = hm.download(), hp.download()
    assert np.array_equal(a.infront, b.infront)
    assert float(np.max(np.abs(a.x - b.x))) < 1e-9
    mg, mp = hm.event_margins(), hp.event_margins()
    for k in KEYS:
        assert 0.0 < mg[k] < 1e300 and 0.0 < mp[k] < 1e300
    hm.close()
    hp.close()
