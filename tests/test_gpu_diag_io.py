"""Device diagnostics and restart files against the oracle.

* calculate_diagnostics (src/diagnostic.f90:9-74) on identical inputs: per-point curvature and
  stretching bit for bit, maxima and minima exact, means within 1e-12 relative (the device sums
  in a fixed parallel order, the reference one point after another).
* pinsert's total_length and avg_sep (src/line.f90:39,95) on identical inputs, with new points
  the sweep reaches again, parallel and serial insertion: within 1e-12 relative.
* ts.log rows (src/output.f90:38-40) of a 20-step run printed every 5 steps: the same text.
* data_dump / data_restore (src/output.f90:85-94, src/initial.f90:151-166): a run resumed from
  a var.dat continues exactly as the uninterrupted run, and the snapshot file equals the
  oracle's for identical state.
"""
import numpy as np
import pytest

from helpers import config0_params, config1_params, rel_err, tangle
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def _holed_state(seed=3, rings=12):
    st = tangle(seed, 0.002, n_rings=rings)
    ends = [k for k in range(1, st.pcount + 1) if st.infront[k - 1] < k]
    st.x[ends[3]:ends[4]] = 0
    st.infront[ends[3]:ends[4]] = 0
    st.behind[ends[3]:ends[4]] = 0
    return st


def _params():
    return config0_params(alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.0, 0.1, 0.4))


def test_diagnostics_identical_inputs():
    from nuvort_b200.api import Handle
    p = _params()
    o = Oracle(p, _holed_state())
    o.step(12)
    full = o.download_full()
    c = o.counters()
    with Handle(p, [full.pcount + 256], states=[]) as h:
        h.upload_full(0, full)
        h.set_clock(0, c.t, c.itime)
        h.calculate_diagnostics()
        o.calculate_diagnostics()
        a, b = h.download_full(), o.download_full()
        assert np.array_equal(a.curv, b.curv) and np.array_equal(a.stretch, b.stretch)
        ra, rb = h.ts_row(), o.ts_row()
    assert ra.live == rb.live and ra.itime == rb.itime and ra.t == rb.t
    for f in ("maxu", "maxdu", "kappa_max", "kappa_min"):
        assert getattr(ra, f) == getattr(rb, f), f
    for f in ("mean_u_sup", "mean_u_mf", "kappa_bar"):
        assert _rel(getattr(ra, f), getattr(rb, f)) <= 1e-12, f


def _moved_state(p, st):
    o = Oracle(p, st)
    o.stage("ghostp")
    o.stage("pmotion")
    return o.download()


@pytest.mark.parametrize("iters", [6, 0])
@pytest.mark.parametrize("revisits", [False, True])
def test_pinsert_lengths_identical_inputs(iters, revisits):
    # revisits: free slots above the inserting points (an emptied last ring) and delta below
    # half the spacing, so the sweep reaches new points and they insert again
    from nuvort_b200.api import Handle
    st = tangle(27, 0.002, n_rings=6)
    if revisits:
        start = st.infront[st.pcount - 1]
        st.x[start - 1:] = 0
        st.infront[start - 1:] = 0
        st.behind[start - 1:] = 0
        p_ins = config0_params(delta=0.0009, overide_timestep_check=True)
    else:
        p_ins = config0_params(delta=0.00185)
    mv = _moved_state(config0_params(), st)
    with Handle(p_ins, [mv.pcount + 8192], states=[mv]) as h:
        h.set_insert_iterations(iters)
        h.set_clock(0, 0.0, 1)
        h.stage("pinsert")
        h.calculate_diagnostics()
        ra = h.ts_row()
        ca = h.counters()
    o = Oracle(p_ins, mv, t=0.0, itime=1)
    o.stage("pinsert")
    o.calculate_diagnostics()
    rb = o.ts_row()
    assert ca.insert_count == o.counters().insert_count > 0
    assert _rel(ra.total_length, rb.total_length) <= 1e-12
    assert _rel(ra.avg_sep, rb.avg_sep) <= 1e-12


def test_ts_rows_of_a_run():
    from nuvort_b200.api import Handle, format_ts_row
    p = config1_params("Tree", delta=0.001)
    st = tangle(1, 0.001, n_points=4096)
    o = Oracle(p, st)
    with Handle(p, [st.pcount + 2048], states=[st]) as h:
        for _ in range(4):
            h.step(5)
            o.step(5)
            h.calculate_diagnostics()
            o.calculate_diagnostics()
            ra, rb = h.ts_row(), o.ts_row()
            assert format_ts_row(ra, 5) == format_ts_row(rb, 5)
            assert (ra.live, ra.recon_count, ra.remove_count, ra.tree_eval) == \
                (rb.live, rb.recon_count, rb.remove_count, rb.tree_eval)
            for f in ("total_length", "avg_sep", "maxu", "maxdu", "mean_u_sup", "mean_u_mf", "kappa_bar",
                      "kappa_max"):
                assert _rel(getattr(ra, f), getattr(rb, f)) <= 1e-9, f


def test_restart_from_dump_continues_exactly(tmp_path):
    from nuvort_b200.api import Handle
    p = config1_params("Tree", delta=0.001)
    st = tangle(2, 0.001, n_points=4096)
    cap = [st.pcount + 2048]
    path = str(tmp_path / "var.dat")
    with Handle(p, cap, states=[st]) as a:
        a.step(25)
        ea, fa, ca = a.events(), a.download_full(), a.counters()
    with Handle(p, cap, states=[st]) as b:
        b.step(12)
        n12 = len(b.events())
        cb = b.counters()
        b.write_dump(0, path)
    with Handle(p, cap) as c:
        c.restore_dump(0, path)
        cc = c.counters()
        assert (cc.itime, cc.t, cc.recon_count, cc.pcount) == (12, cb.t, cb.recon_count, cb.pcount)
        c.step(13)
        ec, fc, cc = c.events(), c.download_full(), c.counters()
    assert ec == ea[n12:] and len(ec) > 0
    assert (cc.itime, cc.t, cc.recon_count) == (ca.itime, ca.t, ca.recon_count)
    for name in ("x", "u", "u1", "u2", "infront", "behind", "u_sup", "u_mf"):
        assert np.array_equal(getattr(fc, name), getattr(fa, name)), name


def test_snapshot_equals_oracle_for_identical_state(tmp_path):
    from nuvort_b200.api import Handle
    p = _params()
    o = Oracle(p, _holed_state(5, 10))
    o.step(8)
    full = o.download_full()
    c = o.counters()
    with Handle(p, [full.pcount + 64]) as h:
        h.upload_full(0, full)
        h.set_clock(0, c.t, c.itime)
        h.calculate_diagnostics()
        o.calculate_diagnostics()
        h.write_snapshot(0, str(tmp_path / "gpu.log"))
        h.write_dump(0, str(tmp_path / "gpu.dat"))
    o.write_snapshot(str(tmp_path / "ref.log"))
    o.write_dump(str(tmp_path / "ref.dat"))
    assert (tmp_path / "gpu.log").read_bytes() == (tmp_path / "ref.log").read_bytes()
    # the dump holds recon_count: the device copy starts from the upload's 0
    from nuvort_b200.api import dump_read_file
    ga, _, gi, gt = dump_read_file(str(tmp_path / "gpu.dat"))
    ra, _, ri, rt = dump_read_file(str(tmp_path / "ref.dat"))
    assert (gi, gt) == (ri, rt)
    from nuvort_b200.abi import FIELDS
    for name in FIELDS:
        assert np.array_equal(getattr(ga, name), getattr(ra, name)), name
