"""Mixed-precision path (FP32 far field, FP64 near field and epilogue) against the plain
FP64 path and the FP64 direct-sum oracle.

Tolerance: relative RMS velocity error <= 1e-6 (sqrt(sum|u_mixed - u_ref|^2 / sum|u_ref|^2)),
the bound the mixed path promises; events over 20 whole steps must equal the plain path's."""
import numpy as np
import pytest

from helpers import config0_params, config1_params, rms_rel, tangle
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL_RMS = 1e-6


def _vel(p, st, extra=512):
    from nuvort_b200.api import Handle
    with Handle(p, [st.pcount + extra], states=[st]) as h:
        u = h.calc_velocity()
        c = h.counters()
    return u, c


@pytest.mark.parametrize("n", [2048, 16384])
def test_mixed_direct_vs_plain_and_oracle(n):
    st = tangle(1, 0.001, n_points=n)
    up, _ = _vel(config1_params("BS", precision="fp64"), st)
    um, _ = _vel(config1_params("BS", precision="mixed"), st)
    e = rms_rel(um, up)
    print("mixed direct rms vs plain", e)
    assert e <= TOL_RMS
    if n <= 2048:
        uo = Oracle(config1_params("BS"), st).calc_velocity()
        assert rms_rel(um, uo) <= TOL_RMS


def test_mixed_direct_config0_small_system():
    st = tangle(0, 0.002, n_rings=8)
    up, _ = _vel(config0_params(), st)
    um, _ = _vel(config0_params(precision="mixed"), st)
    assert rms_rel(um, up) <= TOL_RMS


@pytest.mark.parametrize("theta", [0.4, 0.5])
def test_mixed_tree_vs_plain(theta):
    st = tangle(1, 0.001, n_points=32768)
    up, cp = _vel(config1_params("Tree", tree_theta=theta, precision="fp64"), st)
    um, cm = _vel(config1_params("Tree", tree_theta=theta, precision="mixed"), st)
    e = rms_rel(um, up)
    print("mixed tree rms vs plain", e, cp.tree_eval, cm.tree_eval)
    assert e <= TOL_RMS
    assert abs(cm.tree_tests - cp.tree_tests) <= 1e-6 * cp.tree_tests + 10
    assert abs(cm.tree_eval - cp.tree_eval) <= 1e-5 * cp.tree_eval + 10


def test_mixed_whole_steps_events_match_plain():
    from nuvort_b200.api import Handle
    st = tangle(1, 0.001, n_points=8192)
    ev = []
    for prec in ("fp64", "mixed"):
        with Handle(config1_params("Tree", precision=prec), [st.pcount + 4096], states=[st]) as h:
            h.step(20)
            ev.append(h.events())
    assert len(ev[0]) > 0
    assert ev[0] == ev[1]


def test_mixed_tree_with_root_tests_deferred():
    # every (target, image) root test deferred: those images' partials come from the exact
    # FP64 walk after the root sums, still within the mixed tolerance of the plain path
    from nuvort_b200.api import Handle
    st = tangle(2, 0.001, n_points=4096)
    hp = Handle(config1_params("Tree", tree_theta=0.4), [st.pcount + 512], states=[st])
    up = hp.calc_velocity()
    hm = Handle(config1_params("Tree", tree_theta=0.4, precision="mixed"), [st.pcount + 512], states=[st])
    hm.set_root_band(1e30)
    um = hm.calc_velocity()
    assert rms_rel(um, up) <= TOL_RMS
    hp.close()
    hm.close()


def test_mixed_walk_after_a_relinking_stage_between_build_and_velocity():
    # Stages one by one with pinsert between the tree build and the velocity: the mixed walk
    # refreshes the links its leaf records took at the build (the own-segment test follows
    # the links of the moment, as the FP64 walk does).  delta is above the state's spacing,
    # so pinsert inserts nothing and the refreshed records equal the built ones: the velocity
    # must equal the one computed right after the build, bit for bit.
    from nuvort_b200.api import Handle
    st = tangle(3, 0.001, n_points=4096)
    p = config1_params("Tree", delta=0.0015, precision="mixed")
    with Handle(p, [2 * st.pcount], states=[st]) as h:
        u0 = h.calc_velocity()
    with Handle(p, [2 * st.pcount], states=[st]) as h:
        for s_ in ("ghostp", "construct_tree", "pinsert", "pmotion"):
            h.stage(s_)
        assert h.counters().insert_count == 0
        u1 = h.download().u[: st.pcount]
    assert np.array_equal(u0, u1)


@pytest.mark.parametrize("parts", [1, 2, 8])
@pytest.mark.parametrize("band", [1.0, 1e30])
def test_mixed_tree_central_image_split(parts, band):
    # The central image's walks split over groups of the root's children: the union of the
    # groups' walks is the whole walk, so the opening tests and accepted nodes are the
    # unsplit walk's; only the grouping of the FP32 partial sums and of their FP64 additions
    # changes (both results within the mixed tolerance of the plain path).
    # band 1e30 defers every root test (the exact FP64 fix-up then writes the central image
    # whole and the other groups must hold zeros).
    from nuvort_b200.api import Handle
    st = tangle(1, 0.001, n_points=16384)
    p = config1_params("Tree", tree_theta=0.4, precision="mixed")
    out = {}
    for k in (1, parts):
        with Handle(p, [st.pcount + 512], states=[st]) as h:
            h.set_walk_parts(k)
            h.set_root_band(band)
            u = h.calc_velocity()
            c = h.counters()
            out[k] = (u, c.tree_tests, c.tree_eval)
    (u1, t1, e1), (uk, tk, ek) = out[1], out[parts]
    assert (tk, ek) == (t1, e1)
    assert rms_rel(uk, u1) <= 2e-7
    up, _ = _vel(config1_params("Tree", tree_theta=0.4, precision="fp64"), st)
    assert rms_rel(uk, up) <= TOL_RMS


def test_walk_parts_argument_checked():
    from nuvort_b200.api import Handle, NuvortError
    st = tangle(1, 0.001, n_points=1024)
    with Handle(config1_params("Tree", precision="mixed"), [st.pcount + 64], states=[st]) as h:
        for bad in (-1, 3, 16):
            with pytest.raises(NuvortError):
                h.set_walk_parts(bad)


def test_fp64_stable_form_matches_reference_arithmetic():
    # With a near radius beyond the box every pair of the mixed direct sum takes the FP64
    # path: the reference's skip decision, the value from the cancellation-free form with
    # reciprocals and reciprocal square roots by Newton's iteration.  Its error bound: a few
    # FP64 roundings per term, so every point agrees with the plain path to 1e-13 relative.
    from helpers import rel_err
    from nuvort_b200.api import Handle
    st = tangle(1, 0.001, n_points=2048)
    up, _ = _vel(config1_params("BS", precision="fp64"), st)
    with Handle(config1_params("BS", precision="mixed"), [st.pcount + 64], states=[st]) as h:
        h.set_near_factor(1e9)
        um = h.calc_velocity()
    assert rel_err(um, up).max() <= 1e-13


def test_fp32_guard_arguments():
    from nuvort_b200.api import Handle, NuvortError
    st = tangle(1, 0.001, n_points=1024)
    with Handle(config1_params("Tree", precision="mixed"), [st.pcount + 64], states=[st]) as h:
        h.set_fp32_guards(0.0, 1e-3, 1e-2)  # the angle guard may be off
        for bad in ((-0.1, 1e-3, 1e-2), (0.1, 0.0, 1e-2), (0.1, 1e-3, 2.0)):
            with pytest.raises(NuvortError):
                h.set_fp32_guards(*bad)
