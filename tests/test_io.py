"""Snapshot and restart files on the CPU: the library's host writers against the oracle's
restatement of printf and data_dump (src/output.f90:47-70, 85-94), byte for byte; the reader
(data_restore, src/initial.f90:151-166) back to the same arrays; the layout the MATLAB reader
expects (bin/vortex/vortex_load.m:18-31); and the ts.log row format (src/output.f90:38-40).
No GPU: these run on the host functions of the C ABI."""
import struct

import numpy as np
import pytest

from helpers import config0_params, tangle
from oracle import Oracle


@pytest.fixture(scope="module")
def stepped():
    """An oracle system after 12 steps with mutual friction (u_sup, u_mf set, some slots
    emptied by the topology) and a diagnostics pass (curv, stretch)."""
    p = config0_params(alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.0, 0.1, 0.4))
    st = tangle(3, 0.002, n_rings=12)
    ends = [k for k in range(1, st.pcount + 1) if st.infront[k - 1] < k]  # last slot of each ring
    st.x[ends[3]:ends[4]] = 0  # the fifth ring's slots empty
    st.infront[ends[3]:ends[4]] = 0
    st.behind[ends[3]:ends[4]] = 0
    o = Oracle(p, st)
    o.step(12)
    o.calculate_diagnostics()
    return o


def test_files_match_oracle_writers_byte_for_byte(stepped, tmp_path):
    from nuvort_b200 import api
    o = stepped
    st = o.download_full()
    c = o.counters()
    assert np.count_nonzero(st.infront == 0) > 0 and np.count_nonzero(st.u_mf) > 0 and np.count_nonzero(st.curv) > 0
    api.dump_write_file(st, c.recon_count, c.itime, c.t, str(tmp_path / "lib.dat"))
    o.write_dump(str(tmp_path / "ref.dat"))
    assert (tmp_path / "lib.dat").read_bytes() == (tmp_path / "ref.dat").read_bytes()
    api.snapshot_write_file(st, c.t, str(tmp_path / "lib.log"))
    o.write_snapshot(str(tmp_path / "ref.log"))
    assert (tmp_path / "lib.log").read_bytes() == (tmp_path / "ref.log").read_bytes()


def test_dump_reads_back_every_field(stepped, tmp_path):
    from nuvort_b200 import api
    from nuvort_b200.abi import FIELDS
    o = stepped
    st = o.download_full()
    c = o.counters()
    path = str(tmp_path / "var.dat")
    o.write_dump(path)
    back, recon, itime, t = api.dump_read_file(path)
    assert (recon, itime, t) == (c.recon_count, c.itime, c.t)
    for name in FIELDS:
        assert np.array_equal(getattr(back, name), getattr(st, name)), name
    # the record framing: 4-byte markers around pcount, recon_count, itime, t and f
    raw = open(path, "rb").read()
    n = st.pcount
    assert struct.unpack_from("<iii", raw, 0) == (4, n, 4)
    assert struct.unpack_from("<i", raw, 3 * 12 + 16)[0] == 248 * n
    assert len(raw) == 3 * 12 + 16 + 8 + 248 * n


def test_snapshot_layout_matches_matlab_reader(stepped, tmp_path):
    # the field order of vortex_load.m: time, count, x, y, z, infront, ux, uy, uz,
    # u_mf x/y/z, curvature, stretching
    o = stepped
    st = o.download_full()
    path = str(tmp_path / "var0001.log")
    o.write_snapshot(path)
    raw = open(path, "rb").read()
    t, n = struct.unpack_from("<di", raw, 0)
    assert t == o.counters().t and n == st.pcount
    off = 12
    def take(dt, k):
        nonlocal off
        a = np.frombuffer(raw, dtype=dt, count=k, offset=off)
        off += a.nbytes
        return a
    for c in range(3):
        assert np.array_equal(take("<f8", n), st.x[:, c])
    assert np.array_equal(take("<i4", n), st.infront)
    for c in range(3):
        assert np.array_equal(take("<f8", n), st.u[:, c])
    for c in range(3):
        assert np.array_equal(take("<f8", n), st.u_mf[:, c])
    assert np.array_equal(take("<f8", n), st.curv)
    assert np.array_equal(take("<f8", n), st.stretch)
    assert off == len(raw)


def test_dump_reader_refusals(stepped, tmp_path):
    from nuvort_b200 import api
    from nuvort_b200.abi import NV_ERR_IO
    path = tmp_path / "var.dat"
    stepped.write_dump(str(path))
    raw = path.read_bytes()
    (tmp_path / "short.dat").write_bytes(raw[:-9])
    with pytest.raises(api.NuvortError) as e:
        api.dump_read_file(str(tmp_path / "short.dat"))
    assert e.value.code == NV_ERR_IO
    pinned = bytearray(raw)
    first = 3 * 12 + 16 + 4  # start of f's first element
    pinned[first + 228:first + 232] = struct.pack("<i", -1)  # wpinned(1) = -1
    pinned[first + 240:first + 244] = struct.pack("<i", 1)  # pinnedi = .true.
    (tmp_path / "pinned.dat").write_bytes(bytes(pinned))
    st, _, _, _ = api.dump_read_file(str(tmp_path / "pinned.dat"))  # the reader keeps the pinned fields
    assert st.pinnedi[0] == 1 and st.pinnedb[0] == 0 and list(st.wpinned[0]) == [-1, 0, 0]
    assert not st.pinnedi[1:].any() and not st.wpinned[1:].any()
    with pytest.raises(api.NuvortError) as e:
        api.dump_read_file(str(tmp_path / "missing.dat"))
    assert e.value.code == NV_ERR_IO


def test_ts_row_format_as_gfortran_writes_it():
    from nuvort_b200 import api
    from nuvort_b200.abi import NvTsRow
    r = NvTsRow(itime=20, live=600, recon_count=3, remove_count=5, tree_eval=123456, t=4e-4, delta=0.002,
                avg_sep=0.0019, total_length=1.234567, maxu=12.3456, maxdu=0.5, kappa_bar=321.456)
    line = api.format_ts_row(r, 10)
    assert line == ("  0002    0.0004000       600            3            0 0.9500     1.234567     12.34560"
                    "      0.50000    321.46            5       123456")
    widths = [6, 13, 10, 13, 13, 7, 13, 13, 13, 10, 13, 13]
    assert len(line) == sum(widths)
    r.kappa_bar = 1e9  # does not fit f10.2: ten asterisks
    r.avg_sep = float("inf")
    line = api.format_ts_row(r, 10)
    assert line[6 + 13 + 10 + 13 + 13:][:7] == "    Inf"
    assert "*" * 10 in line


def test_oracle_diagnostics_known_values():
    # a single circular ring: curvature 1/R at every point (to the finite-difference error),
    # stretching u . s'' from the stored velocities, live count and the empty-mask minimum
    from nuvort_b200.rings import single_ring
    R = 0.02
    st = single_ring(R, 120)
    p = config0_params()
    o = Oracle(p, st)
    o.calculate_diagnostics()
    row = o.ts_row()
    assert row.live == 120
    assert abs(row.kappa_bar - 1 / R) < 1e-3 / R and abs(row.kappa_max - 1 / R) < 1e-3 / R
    assert row.maxu == 0.0 and row.mean_u_sup == 0.0  # no velocity pass yet
