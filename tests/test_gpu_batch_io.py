"""nv_upload_many / nv_download_many against one nv_upload / nv_download per system: the
same device state and the same host arrays bit for bit, a rejected link check that changes
no system, the all-or-none rule for optional arrays, page-locked host arrays, and solid-wall
systems going through the single calls."""
import numpy as np
import pytest

from helpers import config0_params, config1_params, tangle

pytestmark = pytest.mark.gpu


def _ensemble(n=6):
    p = config1_params("Tree")
    sts = [tangle(40 + i, 0.001, n_points=600 + 170 * i) for i in range(n)]
    return [p] * n, sts


def _same(a, b):
    for f in ("x", "u", "u1", "u2", "ghosti", "ghostb", "infront", "behind", "closest", "closestd"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_batched_transfers_equal_single_calls():
    from nuvort_b200.api import Handle
    ps, sts = _ensemble()
    caps = [s.pcount + 400 for s in sts]
    with Handle(ps, caps) as h1, Handle(ps, caps) as h2:
        for s, st in enumerate(sts):
            h1.upload(s, st)
        h2.upload_many(sts)
        h1.step(3)
        h2.step(3)
        singles = [h1.download(s) for s in range(len(sts))]
        many = h2.download_many()
        for a, b in zip(singles, many):
            _same(a, b)
        # round trip of the stepped state through the batched calls, in a different order
        order = [3, 0, 5, 1, 4, 2]
        h2.upload_many([many[s] for s in order], systems=order)
        _same(h2.download(3), many[3])
        c1, c2 = h1.counters(2), h2.counters(2)
        assert c2.live == int(np.count_nonzero(many[2].infront)) and c2.itime == c1.itime


def test_rejected_batch_changes_nothing():
    from nuvort_b200.abi import NV_ERR_ARG
    from nuvort_b200.api import Handle, NuvortError
    ps, sts = _ensemble(3)
    caps = [s.pcount + 64 for s in sts]
    with Handle(ps, caps, states=sts) as h:
        before = h.download_many()
        bad = [s.copy() for s in sts]
        bad[2].infront[5] = bad[2].pcount + 3  # out of range in the last system only
        with pytest.raises(NuvortError) as e:
            h.upload_many(bad)
        assert e.value.code == NV_ERR_ARG and "system 2" in str(e.value)
        for a, b in zip(before, h.download_many()):
            _same(a, b)
        mixed = [s.copy() for s in sts]
        mixed[1].u = None  # u given for some systems only
        with pytest.raises(NuvortError):
            h.upload_many(mixed)
        with pytest.raises(NuvortError):
            h.upload_many(sts[:2], systems=[1, 1])


def test_page_locked_host_arrays():
    from nuvort_b200 import api
    from nuvort_b200.abi import State
    ps, sts = _ensemble(4)
    caps = [s.pcount + 64 for s in sts]
    bufs = [State.empty(c) for c in caps]
    arrays = [a for b in bufs for a in (b.x, b.infront, b.behind)]
    for a in arrays:
        api.host_register(a)
    try:
        with api.Handle(ps, caps, states=sts) as h:
            got = h.download_many(bufs, fields=("x", "infront", "behind"))
            for a, st in zip(got, sts):
                assert np.array_equal(a.x, st.x) and np.array_equal(a.infront, st.infront)
    finally:
        for a in arrays:
            api.host_unregister(a)


def test_solid_wall_systems_one_by_one():
    from nuvort_b200.api import Handle
    from nuvort_b200.rings import half_loop
    p = config0_params(boundary_x="solid")
    st = half_loop(40, 0.002)
    with Handle([p, p], [st.pcount + 64] * 2) as h:
        h.upload_many([st, st])
        for s in (0, 1):
            d = h.download(s)
            assert np.array_equal(d.pinnedi, st.pinnedi) and np.array_equal(d.wpinned, st.wpinned)
            assert np.array_equal(d.x, st.x)


def test_batch_buffers_round_trip():
    from nuvort_b200.api import BatchBuffers, Handle
    ps, sts = _ensemble(5)
    caps = [s.pcount + 300 for s in sts]
    with Handle(ps, caps, states=sts) as h:
        hb = BatchBuffers(h)
        try:
            hb.download()
            assert hb.pcounts() == [s.pcount for s in sts]
            assert hb.live_points() == sum(int(np.count_nonzero(s.infront)) for s in sts)
            for s, st in enumerate(sts):
                assert np.array_equal(hb.rows(s, "x"), st.x)
            h.step(2)
            hb.download()
            ref = h.download_many()
            hb.upload()  # the same state back: nothing changes
            for s, r in enumerate(ref):
                assert np.array_equal(hb.rows(s, "infront"), r.infront)
                assert np.array_equal(h.download(s).x, r.x)
            # a packed upload with a bad link in one system changes nothing
            from nuvort_b200.api import NuvortError
            hb.rows(3, "infront")[7] = hb.pcounts()[3] + 5
            with pytest.raises(NuvortError):
                hb.upload()
            for s, r in enumerate(ref):
                assert np.array_equal(h.download(s).infront, r.infront)
        finally:
            hb.close()
