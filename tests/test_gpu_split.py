"""One tangle's velocity pass split over ranks (nv_set_walk_range, nv_velocity_pack/unpack,
nv_step_velocity/nv_step_finish): two handles on one GPU, each computing half of the walk
order and taking the other half's velocities between the two halves of the step, stay
equal bit for bit to one handle running nv_step -- positions, links, events -- in both
precisions.  (The exchange here goes through the host program; between GPUs it is the
all-gather of nuvort_b200.dist.TangleSplit.)"""
import numpy as np
import pytest

from helpers import config1_params, tangle
from nuvort_b200.dist import split_ranges, walk_range

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_split_step_equals_one_gpu(precision):
    import torch
    from nuvort_b200.api import Handle
    p = config1_params("Tree", precision=precision)
    st = tangle(7, 0.001, n_points=8192)
    cap = [st.pcount + 4096]
    hs = [Handle(p, cap, states=[st]) for _ in range(2)]
    ref = Handle(p, cap, states=[st])
    try:
        for _ in range(6):
            live = hs[0].counters(0).live
            assert live == hs[1].counters(0).live == ref.counters(0).live
            rg = split_ranges(live, 2)
            for h, (lo, hi) in zip(hs, rg):
                h.set_walk_range(0, *walk_range(lo, hi, cap[0]))
                h.step_velocity()
            bufs = []
            for h, (lo, hi) in zip(hs, rg):
                # (no fill kernel on torch's stream: the pack runs on the library's own stream)
                b = torch.empty((hi - lo, 3), dtype=torch.float64, device="cuda")
                h.velocity_pack(0, lo, hi - lo, b.data_ptr())
                bufs.append(b)
            torch.cuda.synchronize()
            for r, h in enumerate(hs):
                o = 1 - r
                lo, hi = rg[o]
                h.velocity_unpack(0, lo, hi - lo, bufs[o].data_ptr())
                h.step_finish()
            ref.step(1)
        a, b, c = hs[0].download(), hs[1].download(), ref.download()
        for f in ("x", "u", "u1", "u2", "infront", "behind"):
            assert np.array_equal(getattr(a, f), getattr(c, f)), f
            assert np.array_equal(getattr(b, f), getattr(c, f)), f
        assert hs[0].events() == ref.events() == hs[1].events()
    finally:
        for h in hs + [ref]:
            h.close()


def test_walk_range_arguments():
    from nuvort_b200.abi import NV_ERR_ARG, NV_ERR_UNSUPPORTED
    from nuvort_b200.api import Handle, NuvortError
    from helpers import config0_params
    st = tangle(7, 0.001, n_points=1024)
    with Handle(config1_params("Tree"), [st.pcount + 64], states=[st]) as h:
        for lo, hi in ((0, 33), (1, 10), (2, 33), (33, 1)):  # below 1, ends off a warp boundary, reversed
            with pytest.raises(NuvortError) as e:
                h.set_walk_range(0, lo, hi)
            assert e.value.code == NV_ERR_ARG
        h.set_walk_range(0, 1, st.pcount + 65)  # hi = cap + 1
        h.set_walk_range(0, 33, 513)
    with Handle(config0_params(), [st.pcount + 64], states=[st]) as h:  # direct sum: no walk order
        with pytest.raises(NuvortError) as e:
            h.set_walk_range(0, 1, 33)
        assert e.value.code == NV_ERR_UNSUPPORTED
