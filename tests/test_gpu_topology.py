"""Topology stages on the GPU against the oracle.

Identical-input tests upload one state to both sides and run a single stage: every slot,
link, ghost and event must agree bit for bit (the stage's arithmetic is one rounding per
operation on both sides).  The whole-step test runs the full time loop on both sides;
positions then drift only by the ulp-level difference of the device log() in the local
term, and the event logs must be identical."""
import numpy as np
import pytest

from helpers import config0_params, small_rings, tangle
from nuvort_b200.abi import NV_ERR_CAPACITY, State
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _moved_state(p, st, steps=1):
    """Oracle state after ghostp+pmotion: positions moved, ghosts still the step-start ones."""
    o = Oracle(p, st)
    for _ in range(steps):
        o.stage("ghostp")
        o.stage("pmotion")
    return o.download()


def _assert_same(a: State, b: State):
    assert a.pcount == b.pcount
    for name in ("x", "u", "u1", "u2", "ghosti", "ghostb", "infront", "behind"):
        assert np.array_equal(getattr(a, name), getattr(b, name)), name


def _run_stage(p, st, stages, cap_extra=512, insert_iterations=None, diag=None):
    from nuvort_b200.api import Handle
    h = Handle(p, [st.pcount + cap_extra], states=[st])
    if insert_iterations is not None:
        h.set_insert_iterations(insert_iterations)
    h.set_clock(0, 0.0, 1)
    o = Oracle(p, st, t=0.0, itime=1)
    for s in stages:
        h.stage(s)
        o.stage(s)
    a, b = h.download(), o.download()
    ea, eb = h.events(), o.events()
    ca, cb = h.counters(), o.counters()
    # the device keeps the live count through the stage's events (no download needed)
    assert ca.live == int(np.count_nonzero(a.infront)) and cb.live == int(np.count_nonzero(b.infront))
    if diag is not None:
        diag.extend(h.diagnostics(0))
    h.close()
    return a, b, ea, eb, ca, cb


def test_pinsert_identical_inputs():
    st = tangle(21, 0.002, n_rings=10)
    p = config0_params()
    mv = _moved_state(p, st)
    p_ins = config0_params(delta=0.00185)  # many chords now exceed delta
    a, b, ea, eb, ca, cb = _run_stage(p_ins, mv, ["pinsert"], cap_extra=4096)
    assert len(eb) > 20
    assert ea == eb
    _assert_same(a, b)
    assert ca.insert_count == cb.insert_count and ca.pcount == cb.pcount


def test_pinsert_fills_empty_slots_then_appends():
    st = tangle(22, 0.002, n_rings=10)
    # empty one ring so insertions reuse its slots first (minloc, line.f90:44-47)
    n0 = 1
    while st.infront[n0 - 1] != 1:
        n0 += 1
    first_ring = n0
    st.x[:first_ring] = 0
    st.infront[:first_ring] = 0
    st.behind[:first_ring] = 0
    p = config0_params()
    mv = _moved_state(p, st)
    a, b, ea, eb, ca, cb = _run_stage(config0_params(delta=0.0018), mv, ["pinsert"], cap_extra=4096)
    assert ea == eb
    _assert_same(a, b)
    assert any(j <= first_ring for (_, k, i, j) in eb if k == 1)


def test_pinsert_capacity_error():
    from nuvort_b200.api import Handle, NuvortError
    st = tangle(23, 0.002, n_rings=6)
    mv = _moved_state(config0_params(), st)
    h = Handle(config0_params(delta=0.0018), [mv.pcount + 2], states=[mv])
    with pytest.raises(NuvortError) as e:
        h.stage("pinsert")
    assert e.value.code == NV_ERR_CAPACITY
    h.close()


def test_premove_cascade_identical_inputs():
    st = tangle(24, 0.002, n_rings=10)
    p = config0_params()
    mv = _moved_state(p, st)
    p_rm = config0_params(delta=0.004, overide_timestep_check=True)
    a, b, ea, eb, ca, cb = _run_stage(p_rm, mv, ["premove"])
    assert ca.remove_count == cb.remove_count and cb.remove_count > 0
    assert ea == eb
    _assert_same(a, b)


def test_premove_kills_small_loops():
    st = small_rings(25, 8, 6, 0.0025)
    p = config0_params()
    mv = _moved_state(p, st)
    p_rm = config0_params(delta=0.005, overide_timestep_check=True)  # loops fall below 4 points
    a, b, ea, eb, ca, cb = _run_stage(p_rm, mv, ["premove"])
    assert cb.loop_kills > 0
    assert ea == eb
    _assert_same(a, b)


def test_pclose_precon_identical_inputs():
    st = tangle(26, 0.002, n_rings=40)  # dense: rings cross at t=0
    p = config0_params()
    mv = _moved_state(p, st)
    a, b, ea, eb, ca, cb = _run_stage(p, mv, ["pclose", "precon"])
    assert np.array_equal(a.closest, b.closest)
    assert np.array_equal(a.closestd, b.closestd)
    assert cb.recon_count > 0
    assert ea == eb
    _assert_same(a, b)


def test_whole_steps_config0_events_identical():
    from nuvort_b200.api import Handle
    st = tangle(0, 0.002, n_rings=8)
    p = config0_params()
    h = Handle(p, [st.pcount + 512], states=[st])
    o = Oracle(p, st)
    h.step(200)
    o.step(200)
    ev = o.events()
    assert h.events() == ev
    from nuvort_b200.abi import event_digest
    assert h.counters().event_hash == event_digest(ev)  # the device digest of the same sequence
    a, b = h.download(), o.download()
    assert np.array_equal(a.infront, b.infront) and np.array_equal(a.behind, b.behind)
    assert np.max(np.abs(a.x - b.x)) < 1e-12
    ca, cb = h.counters(), o.counters()
    assert (ca.recon_count, ca.remove_count, ca.insert_count) == (cb.recon_count, cb.remove_count, cb.insert_count)
    assert ca.live == cb.live == int(np.count_nonzero(a.infront))
    assert ca.t == cb.t and ca.itime == cb.itime == 200
    h.close()


@pytest.mark.parametrize("iters", [6, 0])
def test_pinsert_new_points_revisited(iters):
    # chords near 0.002 with delta 0.0009: every segment inserts and each new midpoint is
    # itself longer than delta from its infront.  Emptying the last ring puts free slots
    # above the inserting points, so the sweep reaches those new points and inserts again.
    st = tangle(27, 0.002, n_rings=6)
    start = st.infront[st.pcount - 1]  # first slot of the last ring
    st.x[start - 1:] = 0
    st.infront[start - 1:] = 0
    st.behind[start - 1:] = 0
    mv = _moved_state(config0_params(), st)
    p_ins = config0_params(delta=0.0009, overide_timestep_check=True)
    diag = []
    a, b, ea, eb, ca, cb = _run_stage(p_ins, mv, ["pinsert"], cap_extra=8192, insert_iterations=iters, diag=diag)
    assert ea == eb
    _assert_same(a, b)
    # the fixed-point rounds place the new points' own insertions; 0 rounds: serial sweep
    assert diag[2] == (1 if iters == 0 else 0)
    assert iters == 0 or diag[5] > 0


def _ring_slots(st: State):
    """Slots (1-based) of each loop, in order of their lowest slot."""
    seen = np.zeros(st.pcount + 1, bool)
    rings = []
    for s in range(1, st.pcount + 1):
        if seen[s] or st.infront[s - 1] == 0:
            continue
        ring, k = [], s
        while not seen[k]:
            seen[k] = True
            ring.append(k)
            k = int(st.infront[k - 1])
        rings.append(sorted(ring))
    return rings


@pytest.mark.parametrize("iters", [6, 0])
def test_pinsert_interleaved_free_slots_second_order(iters):
    # every third loop emptied: the free slots lie between live loops, so new points are
    # placed just above the loops that create them and the sweep reaches them (and their
    # own new points) between ordinary candidates, many per chunk of 32 candidates
    st = tangle(31, 0.002, n_rings=12)
    for r in _ring_slots(st)[2::3]:
        idx = np.asarray(r) - 1
        for name in ("x", "u", "u1", "u2", "ghosti", "ghostb"):
            getattr(st, name)[idx] = 0
        st.infront[idx] = 0
        st.behind[idx] = 0
    mv = _moved_state(config0_params(), st)
    p_ins = config0_params(delta=0.0009, overide_timestep_check=True)
    diag = []
    a, b, ea, eb, ca, cb = _run_stage(p_ins, mv, ["pinsert"], cap_extra=16384, insert_iterations=iters, diag=diag)
    assert len(eb) > 200
    assert diag[2] == (1 if iters == 0 else 0)
    assert iters == 0 or diag[5] > 100
    assert ea == eb
    _assert_same(a, b)
    assert ca.insert_count == cb.insert_count and ca.pcount == cb.pcount


def _pclose_both(p, st, itime=1):
    """closest/closestd after the pclose stage: cell list, every-slot scan, oracle."""
    from nuvort_b200.api import Handle
    out = []
    for method in (0, 1):
        with Handle(p, [st.pcount + 64], states=[st]) as h:
            h.set_pclose_method(method)
            h.set_clock(0, 0.0, itime)
            h.stage("pclose")
            out.append(h.download())
    o = Oracle(p, st, t=0.0, itime=itime)
    o.stage("pclose")
    out.append(o.download())
    return out


def _assert_same_closest(states):
    a, b, c = states
    for name in ("closest", "closestd"):
        assert np.array_equal(getattr(a, name), getattr(c, name)), name
        assert np.array_equal(getattr(b, name), getattr(c, name)), name


def test_pclose_cell_list_32k_bs():
    # a 32,768-point direct-sum tangle: the cell list, the every-slot scan and the oracle
    # give the same nearest non-neighbour and distance for every point
    st = tangle(1, 0.001, n_points=32768)
    st.closest = np.arange(1, st.pcount + 1, dtype=np.int32)[::-1].copy()  # stale values must be replaced
    st.closestd = np.zeros(st.pcount)
    p = config0_params(delta=0.001, dt=5e-6)
    _assert_same_closest(_pclose_both(p, st))


def test_pclose_cell_list_ties_outside_points_and_no_candidate():
    # squares of 8 points on a 2^-9 cm lattice: many exactly equal distances, so the lowest
    # slot must win; some squares lie partly outside the box (clamped to the edge cells); a
    # small triangle sits far from everything else (a long ring search)
    h9 = 2.0 ** -9
    rng = np.random.default_rng(5)
    xs, nx, pv = [], [], []
    base = 0
    for q in range(60):
        c = rng.integers(-27, 27, 3) * h9
        if q % 10 == 0:
            c[q % 3] = 0.05 + 2 * h9  # beyond the upper face
        ring = [(-1, -1), (0, -1), (1, -1), (1, 0), (1, 1), (0, 1), (-1, 1), (-1, 0)]
        ax = q % 3
        for (u, v) in ring:
            pt = c.copy()
            pt[(ax + 1) % 3] += u * h9
            pt[(ax + 2) % 3] += v * h9
            xs.append(pt)
        n = len(ring)
        nx += [base + (k + 1) % n + 1 for k in range(n)]
        pv += [base + (k - 1) % n + 1 for k in range(n)]
        base += n
    far = np.array([[0.04, 0.04, 0.04], [0.04 + h9, 0.04, 0.04], [0.04, 0.04 + h9, 0.04]])
    xs += list(far)
    nx += [base + 2, base + 3, base + 1]
    pv += [base + 3, base + 1, base + 2]
    x = np.ascontiguousarray(np.array(xs))
    N = len(x)
    st = State(x=x, infront=np.array(nx, np.int32), behind=np.array(pv, np.int32),
               closest=np.full(N, 7, np.int32), closestd=np.zeros(N))
    p = config0_params(delta=0.002)
    res = _pclose_both(p, st)
    _assert_same_closest(res)
    c = res[2]
    assert np.any(c.closestd[:-3] == h9)  # ties exist
    assert np.all(c.closestd < 100)  # the triangle's points find the nearest square point


def test_pclose_no_candidate_keeps_closest():
    # one 3-point loop alone: every other slot is itself or a neighbour
    x = np.array([[0.0, 0.0, 0.0], [0.001, 0.0, 0.0], [0.0, 0.001, 0.0]])
    st = State(x=x, infront=np.array([2, 3, 1], np.int32), behind=np.array([3, 1, 2], np.int32),
               closest=np.array([3, 1, 2], np.int32), closestd=np.zeros(3))
    a, b, c = _pclose_both(config0_params(), st)
    _assert_same_closest((a, b, c))
    assert np.all(c.closestd == 100.0) and np.array_equal(c.closest, [3, 1, 2])
