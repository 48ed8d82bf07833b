"""Solid walls on the GPU against the oracle: the mirror sums of the BS and tree velocities
(src/timestep.f90:201-234, src/tree.f90:321-396), the tree without the segments into the
wall, and whole steps through the pinned-point topology (pinsert and premove skipping pinned
points, pclose not testing them, loop_killer stopping at them, wall_recon cutting filaments
at the walls and clearing wall pairs, enforce_boundary putting pinned points back on their
wall).  Velocities within 1e-12 relative (the plain FP64 path); whole steps with identical
event sequences, links and pinned records, positions within 1e-12."""
import numpy as np
import pytest

from helpers import config0_params, rel_err
from nuvort_b200.abi import NV_EV_CLEAR, NV_EV_WALL
from nuvort_b200.rings import half_loop, lattice, single_ring
from oracle import Oracle

pytestmark = pytest.mark.gpu

TOL = 1e-12
DELTA = 0.002
L = 0.1


def _params(velocity="BS", walls="x", **kw):
    b = {a: ("solid" if a in walls else "periodic") for a in "xyz"}
    extra = dict(tree_theta=0.4) if velocity == "Tree" else {}
    extra.update(kw)
    return config0_params(velocity=velocity, boundary_x=b["x"], boundary_y=b["y"], boundary_z=b["z"], **extra)


def _handle(p, st, extra=512):
    from nuvort_b200.api import Handle
    return Handle(p, [st.pcount + extra], states=[st])


def _velocities(p, st):
    with _handle(p, st) as h:
        ug = h.calc_velocity()
        eg = h.counters().tree_eval
    o = Oracle(p, st)
    uo = o.calc_velocity()
    return ug, uo, eg, o.counters().tree_eval


def _same_state(a, b):
    assert np.array_equal(a.infront, b.infront)
    assert np.array_equal(a.behind, b.behind)
    assert np.array_equal(a.pinnedi, b.pinnedi)
    assert np.array_equal(a.pinnedb, b.pinnedb)
    assert np.array_equal(a.wpinned, b.wpinned)
    assert np.max(np.abs(a.x - b.x)) < 1e-12


@pytest.mark.parametrize("velocity", ["BS", "Tree"])
@pytest.mark.parametrize("walls", ["x", "xyz"])
def test_half_loop_velocity(velocity, walls):
    st = half_loop(60, DELTA)
    ug, uo, eg, eo = _velocities(_params(velocity, walls), st)
    assert rel_err(ug, uo).max() <= TOL
    assert eg == eo


@pytest.mark.parametrize("velocity", ["BS", "Tree"])
def test_lattice_velocity(velocity):
    st = lattice(3, DELTA)  # 19 lines of 67 points from the +z wall to the -z wall
    ug, uo, eg, eo = _velocities(_params(velocity, "z"), st)
    assert rel_err(ug, uo).max() <= TOL
    assert eg == eo


def test_half_loop_z_wall_velocity():
    st = half_loop(50, DELTA, axis=2)
    ug, uo, _, _ = _velocities(_params("BS", "z"), st)
    assert rel_err(ug, uo).max() <= TOL


def test_tree_leaves_out_segments_into_the_wall():
    st = lattice(3, DELTA)
    p = _params("Tree", "z")
    with _handle(p, st) as h:
        h.stage("ghostp")
        h.stage("construct_tree")
        tg = h.tree_dump()
    o = Oracle(p, st)
    o.stage("ghostp")
    o.stage("construct_tree")
    to = o.tree_dump()
    assert len(tg) == len(to)
    for f in ("pos", "width", "cent", "circ", "pcount", "leaf", "first_next"):
        assert np.array_equal(tg[f], to[f]), f
    # no leaf holds a point pinned in front
    leaves = tg["leaf"][tg["pcount"] == 1]
    assert not st.pinnedi[leaves[leaves > 0] - 1].any()


def _ring_at_wall(n=64, R=0.012, gap=0.2 * DELTA):
    """A ring in the x-y plane whose outermost point lies gap inside the +x wall's cut
    distance: wall_recon cuts it at the first reconnection step."""
    return single_ring(R, n, centre=(0.5 * L - R - gap, 0.003, -0.01), normal=(0.0, 0.0, 1.0))


def _with_pinned_fields(st):
    n = st.pcount
    if st.pinnedi is None:
        st.wpinned = np.zeros((n, 3), np.int32)
        st.pinnedi = np.zeros(n, np.int32)
        st.pinnedb = np.zeros(n, np.int32)
    return st


def _append(a, b):
    """States a then b in one system (b's slots shifted by a's count)."""
    from nuvort_b200.abi import State
    a, b = _with_pinned_fields(a), _with_pinned_fields(b)
    off = a.pcount
    sh = lambda v: np.where(v > 0, v + off, 0).astype(np.int32)
    cat = lambda u, v: np.concatenate([u, v]) if u is not None and v is not None else None
    return State(x=cat(a.x, b.x), infront=np.concatenate([a.infront, sh(b.infront)]),
                 behind=np.concatenate([a.behind, sh(b.behind)]), u=cat(a.u, b.u), u1=cat(a.u1, b.u1),
                 u2=cat(a.u2, b.u2), ghosti=cat(a.ghosti, b.ghosti), ghostb=cat(a.ghostb, b.ghostb),
                 closest=np.zeros(off + b.pcount, np.int32), closestd=np.zeros(off + b.pcount, np.float64),
                 wpinned=cat(a.wpinned, b.wpinned), pinnedi=cat(a.pinnedi, b.pinnedi),
                 pinnedb=cat(a.pinnedb, b.pinnedb))


def _wall_arc(ys, xs, wall_x=0.499999999 * L, z=0.02):
    """An open filament on the +x wall: its first point pinned behind, its last pinned in
    front, both on the wall; interior points at the given x."""
    from nuvort_b200.abi import State
    pts = [(wall_x, ys[0], z)] + [(x, y, z) for x, y in zip(xs, ys[1:-1])] + [(wall_x, ys[-1], z)]
    n = len(pts)
    k = np.arange(n)
    w = np.zeros((n, 3), np.int32)
    w[0, 0] = w[-1, 0] = 1
    pi_ = np.zeros(n, np.int32)
    pb_ = np.zeros(n, np.int32)
    pi_[-1] = 1
    pb_[0] = 1
    z3 = lambda: np.zeros((n, 3))
    return State(x=np.array(pts, np.float64), infront=np.minimum(k + 2, n).astype(np.int32),
                 behind=np.maximum(k, 1).astype(np.int32), u=z3(), u1=z3(), u2=z3(), ghosti=z3(), ghostb=z3(),
                 closest=np.zeros(n, np.int32), closestd=np.zeros(n, np.float64), wpinned=w, pinnedi=pi_,
                 pinnedb=pb_)


def _steps(p, st, n, extra=512):
    with _handle(p, st, extra) as h:
        o = Oracle(p, st)
        h.step(n)
        o.step(n)
        eg, eo = h.events(), o.events()
        a, b = h.download(), o.download()
        cg, co = h.counters(), o.counters()
    return eg, eo, a, b, cg, co


def test_whole_steps_wall_cut_and_wall_pairs():
    # a ring cut at the +x wall, a two-point wall pair (cleared by wall_recon's clean-up) and
    # a three-point arc whose middle point premove removes (its ends then cleared as a pair)
    ring = _ring_at_wall()
    pair = _wall_arc([-0.02, -0.02 + 0.5 * DELTA], [])
    arc = _wall_arc([0.01, 0.0, 0.01 + 0.6 * DELTA], [0.5 * L - 0.6 * DELTA])
    arc.x[1, 1] = 0.01 + 0.3 * DELTA
    st = _append(_append(ring, pair), arc)
    p = _params("BS", "x", alpha=(0.1, 0.01), normal_velocity="xflow", norm_vel_xflow=0.3)
    eg, eo, a, b, cg, co = _steps(p, st, 30)
    assert eg == eo
    kinds = [e[1] for e in eo]
    assert kinds.count(NV_EV_WALL) >= 1 and kinds.count(NV_EV_CLEAR) >= 2
    _same_state(a, b)
    assert cg.wall_recon_count == co.wall_recon_count >= 1
    assert cg.live == np.count_nonzero(b.infront)
    # pinned points sit on their wall after enforce_boundary
    pinned = (b.pinnedi + b.pinnedb) > 0
    assert pinned.any() and np.all(np.abs(b.x[pinned, 0]) == 0.499999999 * L)


@pytest.mark.parametrize("velocity", ["BS", "Tree"])
def test_whole_steps_lattice(velocity):
    # 7 lines; interior points moved along the line by up to 0.45 spacings, delta 0.0019: the
    # first steps insert and remove points along every line, next to the pinned ends too
    st = lattice(2, DELTA)
    inner = (st.pinnedi + st.pinnedb) == 0
    st.x[inner, 2] += np.random.default_rng(7).uniform(-0.45, 0.45, inner.sum()) * (L / 66)
    p = _params(velocity, "z", delta=0.0019, overide_timestep_check=True, alpha=(0.1, 0.01),
                normal_velocity="shear_xflow", norm_vel_xflow=0.5, norm_shear_omega=500.0)
    eg, eo, a, b, cg, co = _steps(p, st, 25)
    assert eg == eo and len(eo) > 100
    _same_state(a, b)
    assert cg.insert_count == co.insert_count and cg.remove_count == co.remove_count


@pytest.mark.parametrize("velocity", ["BS", "Tree"])
def test_whole_steps_all_walls(velocity):
    # a half loop on the +x wall and a ring cut at the +y wall, in a box with six walls
    ring = single_ring(0.008, 40, centre=(0.0, 0.5 * L - 0.008 - 0.15 * 0.0016, 0.01), normal=(1.0, 0.0, 0.0))
    st = _append(half_loop(40, DELTA), ring)
    p = _params(velocity, "xyz", delta=0.0016, overide_timestep_check=True, alpha=(0.1, 0.01),
                normal_velocity="xflow", norm_vel_xflow=-0.5)
    eg, eo, a, b, _, _ = _steps(p, st, 25)
    assert eg == eo
    assert [e[1] for e in eo].count(NV_EV_WALL) >= 1
    _same_state(a, b)


def test_dump_round_trip_keeps_pinned_records(tmp_path):
    from nuvort_b200.abi import NV_ERR_ARG
    from nuvort_b200.api import Handle, NuvortError
    st = half_loop(40, DELTA)
    p = _params("BS", "x")
    path = str(tmp_path / "var.dat")
    with _handle(p, st) as h:
        h.step(3)
        h.write_dump(0, path)
        before = h.download()
    with Handle(p, [st.pcount + 512]) as h2:
        h2.restore_dump(0, path)
        _same_state(h2.download(), before)
    with Handle(config0_params(), [st.pcount + 512]) as h3:  # no solid wall: refused
        with pytest.raises(NuvortError) as e:
            h3.restore_dump(0, path)
        assert e.value.code == NV_ERR_ARG
