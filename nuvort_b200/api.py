"""Python binding of libnuvort_gpu.so (the C ABI in include/nuvort_gpu.h).

The stage methods mirror the reference's module procedures called from its time loop
(src/run.f90:26-64): ``ghostp``, ``construct_tree``, ``pmotion``, ``pinsert``, ``pclose``,
``precon``, ``premove``, ``enforce_boundary``, ``empty_tree``; ``step`` runs whole steps.
Errors the reference reports through ``fatal_error`` + ``stop`` (src/cdata.f90:245-255)
raise :class:`NuvortError` with the library's status code.

There is no CPU fallback: if the CUDA library is missing this module raises on load.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional, Sequence

import numpy as np

from .abi import (ERR_NAMES, NV_OK, NvCounters, NvEvent, NvFullState, NvHostState, NvParams, NvTreeNode, NvTsRow,
                  State, tree_nodes_to_numpy)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libnuvort_gpu.so")

_lib = None

STAGES = ("ghostp", "construct_tree", "pmotion", "pinsert", "pclose", "precon", "wall_recon", "premove",
          "enforce_boundary", "empty_tree", "end_step")
STATE_FIELDS = ("x", "infront", "behind", "u", "u1", "u2", "ghosti", "ghostb", "closest", "closestd", "wpinned",
                "pinnedi", "pinnedb")
STAGE_TIMES = ("ghost", "tree", "velocity", "ab3", "topology", "step", "insert", "close", "recon", "remove")


class NuvortError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Load the CUDA library (built in-tree by nuvort_b200.build); fail loudly if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"libnuvort_gpu.so not found at {LIB_PATH}; run `python -m nuvort_b200.build`")
    L = C.CDLL(LIB_PATH)
    P, vp, i32 = C.POINTER, C.c_void_p, C.c_int32
    L.nv_params_default.argtypes = [P(NvParams)]
    L.nv_read_run_file.argtypes = [C.c_char_p, P(NvParams)]
    L.nv_check_params.argtypes = [P(NvParams)]
    L.nv_create.argtypes = [P(NvParams), i32, P(i32), i32, P(vp)]
    L.nv_destroy.argtypes = [vp]
    L.nv_upload.argtypes = [vp, i32, P(NvHostState)]
    L.nv_download.argtypes = [vp, i32, P(NvHostState), i32]
    L.nv_set_clock.argtypes = [vp, i32, C.c_double, i32]
    L.nv_counters_get.argtypes = [vp, i32, P(NvCounters)]
    L.nv_events_get.argtypes = [vp, i32, P(NvEvent), i32, P(i32)]
    for name in STAGES:
        getattr(L, "nv_" + name).argtypes = [vp]
    L.nv_step.argtypes = [vp, i32]
    L.nv_calc_velocity.argtypes = [vp, i32, P(C.c_double)]
    L.nv_stage_times.argtypes = [vp, P(C.c_double), i32]
    L.nv_sync.argtypes = [vp]
    L.nv_last_error.restype = C.c_char_p
    L.nv_version.restype = C.c_char_p
    L.nv_tree_dump.argtypes = [vp, i32, P(NvTreeNode), i32, P(i32)]
    L.nv_set_timing.argtypes = [vp, i32]
    L.nv_set_near_factor.argtypes = [vp, C.c_double]
    L.nv_set_insert_iterations.argtypes = [vp, C.c_int32]
    L.nv_set_fp32_guards.argtypes = [vp, C.c_double, C.c_double, C.c_double]
    L.nv_set_root_band.argtypes = [vp, C.c_double]
    L.nv_set_walk_parts.argtypes = [vp, C.c_int32]
    L.nv_set_event_margins.argtypes = [vp, C.c_int32]
    L.nv_upload_many.argtypes = [vp, i32, P(i32), P(NvHostState)]
    L.nv_download_many.argtypes = [vp, i32, P(i32), P(NvHostState), P(i32)]
    L.nv_upload_packed.argtypes = [vp, P(NvHostState), P(i32)]
    L.nv_set_walk_range.argtypes = [vp, i32, i32, i32]
    L.nv_velocity_pack.argtypes = [vp, i32, i32, i32, vp]
    L.nv_velocity_unpack.argtypes = [vp, i32, i32, i32, vp]
    L.nv_step_velocity.argtypes = [vp]
    L.nv_step_finish.argtypes = [vp]
    L.nv_download_packed.argtypes = [vp, P(NvHostState), C.c_int64, P(i32)]
    L.nv_host_register.argtypes = [vp, C.c_size_t]
    L.nv_host_unregister.argtypes = [vp]
    L.nv_event_margins_get.argtypes = [vp, i32, P(C.c_double)]
    L.nv_set_direct_split.argtypes = [vp, C.c_int32]
    L.nv_set_pclose_method.argtypes = [vp, C.c_int32]
    L.nv_step_launches.argtypes = [vp, P(i32)]
    L.nv_measure_fp64_peak.argtypes = [i32, P(C.c_double)]
    L.nv_measure_fp32_peak.argtypes = [i32, P(C.c_double)]
    L.nv_diagnostics.argtypes = [vp, i32, P(C.c_int64), i32]
    L.nv_calc_velocity_direct_at.argtypes = [vp, i32, P(i32), i32, P(C.c_double)]
    L.nv_set_normal_fluid_noise.argtypes = [vp, i32, P(C.c_double), i32]
    L.nv_set_normal_fluid_grid.argtypes = [vp, i32, P(C.c_double), i32, i32, i32, P(C.c_double)]
    L.nv_calculate_diagnostics.argtypes = [vp]
    L.nv_ts_row_get.argtypes = [vp, i32, P(NvTsRow)]
    L.nv_format_ts_row.argtypes = [P(NvTsRow), i32, C.c_char_p, i32]
    L.nv_download_full.argtypes = [vp, i32, P(NvFullState), i32]
    L.nv_upload_full.argtypes = [vp, i32, P(NvFullState)]
    L.nv_write_snapshot.argtypes = [vp, i32, C.c_char_p]
    L.nv_write_dump.argtypes = [vp, i32, C.c_char_p]
    L.nv_restore_dump.argtypes = [vp, i32, C.c_char_p]
    L.nv_snapshot_write_file.argtypes = [P(NvFullState), C.c_double, C.c_char_p]
    L.nv_dump_write_file.argtypes = [P(NvFullState), i32, i32, C.c_double, C.c_char_p]
    L.nv_dump_read_file.argtypes = [C.c_char_p, P(NvFullState), i32, P(i32), P(i32), P(i32), P(C.c_double)]
    _lib = L
    return L


def _check(rc: int):
    if rc != NV_OK:
        raise NuvortError(rc, lib().nv_last_error().decode())


def host_register(a: np.ndarray):
    """Page-lock a C-contiguous host array (cudaHostRegister) for asynchronous full-speed copies."""
    _check(lib().nv_host_register(C.c_void_p(a.ctypes.data), C.c_size_t(a.nbytes)))


def host_unregister(a: np.ndarray):
    _check(lib().nv_host_unregister(C.c_void_p(a.ctypes.data)))


class BatchBuffers:
    """Host arrays of every system of a handle, packed as nv_upload_packed / nv_download_packed
    take them (system s's rows follow system s-1's), page-locked, with the C state record
    built once: a transfer of all systems is one call and one copy per array."""

    FIELDS3 = ("x", "u", "u1", "u2", "ghosti", "ghostb")

    def __init__(self, handle: "Handle", fields: Sequence[str] = ("x", "u", "u1", "u2", "infront", "behind")):
        self.handle = handle
        self.n = handle.nsys
        self.cap_rows = int(sum(handle.capacity))
        self.arrays = {}
        for f in fields:
            if f in self.FIELDS3:
                self.arrays[f] = np.zeros((self.cap_rows, 3), np.float64)
            elif f == "closestd":
                self.arrays[f] = np.zeros(self.cap_rows, np.float64)
            else:
                self.arrays[f] = np.zeros(self.cap_rows, np.int32)
        for a in self.arrays.values():
            host_register(a)
        self.rec = NvHostState()
        self.rec.pcount = 0
        for f, a in self.arrays.items():
            setattr(self.rec, f, C.cast(a.ctypes.data, C.POINTER(C.c_double if a.dtype == np.float64 else C.c_int32)))
        self.pc = (C.c_int32 * self.n)()

    def download(self):
        _check(lib().nv_download_packed(self.handle.h, C.byref(self.rec), self.cap_rows, self.pc))

    def upload(self):
        _check(lib().nv_upload_packed(self.handle.h, C.byref(self.rec), self.pc))

    def pcounts(self) -> List[int]:
        return list(self.pc)

    def rows(self, sys: int, field: str) -> np.ndarray:
        """System sys's rows of a field (a view)."""
        o = int(sum(self.pc[:sys]))
        return self.arrays[field][o:o + self.pc[sys]]

    def live_points(self) -> int:
        return int(np.count_nonzero(self.arrays["infront"][:self.rec.pcount]))

    def bytes_of(self, fields: Sequence[str]) -> int:
        """Bytes that one transfer of the given fields moves."""
        n = self.rec.pcount
        return int(sum(n * self.arrays[f].itemsize * (3 if f in self.FIELDS3 else 1) for f in fields))

    def close(self):
        for a in self.arrays.values():
            host_unregister(a)
        self.arrays = {}


def version() -> str:
    return lib().nv_version().decode()


def read_run_file(path: str, params: Optional[NvParams] = None) -> NvParams:
    p = params if params is not None else NvParams()
    if params is None:
        _check(lib().nv_params_default(C.byref(p)))
    _check(lib().nv_read_run_file(path.encode(), C.byref(p)))
    return p


def measure_fp64_peak(device: int = 0) -> float:
    """FP64 FMA throughput of the device in TFLOP/s (the FP64 CUDA-core roofline peak)."""
    v = C.c_double()
    _check(lib().nv_measure_fp64_peak(int(device), C.byref(v)))
    return v.value


def measure_fp32_peak(device: int = 0) -> float:
    """FP32 FMA throughput of the device in TFLOP/s."""
    v = C.c_double()
    _check(lib().nv_measure_fp32_peak(int(device), C.byref(v)))
    return v.value


def check_params(p: NvParams):
    _check(lib().nv_check_params(C.byref(p)))


def format_ts_row(row: NvTsRow, shots: int = 1) -> str:
    """The data/ts.log line print_info writes for this row (src/output.f90:38-40)."""
    buf = C.create_string_buffer(256)
    _check(lib().nv_format_ts_row(C.byref(row), int(shots), buf, 256))
    return buf.value.decode()


def snapshot_write_file(st: State, t: float, path: str):
    """printf's data/var%04d.log stream file (src/output.f90:47-70) from host arrays."""
    c = st.to_full_c()
    _check(lib().nv_snapshot_write_file(C.byref(c), float(t), path.encode()))


def dump_write_file(st: State, recon_count: int, itime: int, t: float, path: str):
    """data_dump's data/var.dat (src/output.f90:85-94) from host arrays."""
    c = st.to_full_c()
    _check(lib().nv_dump_write_file(C.byref(c), int(recon_count), int(itime), float(t), path.encode()))


def dump_read_file(path: str):
    """(State with every kept field, recon_count, itime, t) of a var.dat (src/initial.f90:151-166)."""
    n, rc_, it, t = C.c_int32(), C.c_int32(), C.c_int32(), C.c_double()
    _check(lib().nv_dump_read_file(path.encode(), None, 0, C.byref(n), C.byref(rc_), C.byref(it), C.byref(t)))
    st = State.empty_full(max(n.value, 1))
    c = st.to_full_c()
    _check(lib().nv_dump_read_file(path.encode(), C.byref(c), max(n.value, 1), C.byref(n), C.byref(rc_),
                                   C.byref(it), C.byref(t)))
    return st.trimmed(n.value), rc_.value, it.value, t.value


class Handle:
    """A device-resident ensemble of filament systems (one system is the common case)."""

    def __init__(self, params, capacity: Sequence[int], device: int = 0,
                 states: Optional[Sequence[State]] = None):
        plist = list(params) if isinstance(params, (list, tuple)) else [params]
        n = len(plist)
        if len(capacity) != n:
            raise ValueError("one capacity per system")
        arr = (NvParams * n)(*plist)
        caps = (C.c_int32 * n)(*[int(c) for c in capacity])
        h = C.c_void_p()
        _check(lib().nv_create(arr, n, caps, int(device), C.byref(h)))
        self.h = h
        self.nsys = n
        self.capacity = [int(c) for c in capacity]
        self.params = plist
        if states is not None:
            for s, st in enumerate(states):
                self.upload(s, st)

    def close(self):
        if getattr(self, "h", None):
            lib().nv_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- state -------------------------------------------------------------------------
    def upload(self, sys: int, st: State, t: Optional[float] = None, itime: Optional[int] = None):
        cst = st.to_c()
        _check(lib().nv_upload(self.h, int(sys), C.byref(cst)))
        if t is not None or itime is not None:
            c = self.counters(sys)
            self.set_clock(sys, c.t if t is None else t, c.itime if itime is None else itime)

    def download(self, sys: int = 0, out: Optional[State] = None, fields: Optional[Sequence[str]] = None) -> State:
        """The system's state.  out: a State whose arrays (capacity rows, C-contiguous float64 /
        int32) are filled in place, as a caller's persistent host arrays would be; the result's
        arrays are views of them.  fields: the names to fetch (default: all)."""
        cap = self.capacity[sys]
        st = out if out is not None else State.empty(cap)
        if fields is not None:
            st = State(**{f: (getattr(st, f) if f in fields else None) for f in STATE_FIELDS})
        for f in STATE_FIELDS:
            a = getattr(st, f)
            if a is not None and (a.shape[0] < cap or not a.flags.c_contiguous):
                raise ValueError(f"download: {f} must be C-contiguous with {cap} rows")
        cst = st.to_c()
        _check(lib().nv_download(self.h, int(sys), C.byref(cst), cap))
        return st.trimmed(cst.pcount)

    def upload_many(self, states: Sequence[State], systems: Optional[Sequence[int]] = None):
        """nv_upload of every (system, state) pair at once (default systems 0..len-1)."""
        systems = list(range(len(states))) if systems is None else list(systems)
        cs = (NvHostState * max(len(states), 1))(*[st.to_c() for st in states])
        sy = (C.c_int32 * max(len(systems), 1))(*systems)
        _check(lib().nv_upload_many(self.h, len(states), sy, cs))

    def download_many(self, outs: Optional[Sequence[State]] = None, fields: Optional[Sequence[str]] = None,
                      systems: Optional[Sequence[int]] = None) -> List[State]:
        """nv_download of several systems at once; outs as in download (one State per system)."""
        systems = list(range(self.nsys)) if systems is None else list(systems)
        caps = [self.capacity[s] for s in systems]
        sts = []
        for i, s in enumerate(systems):
            st = outs[i] if outs is not None else State.empty(caps[i])
            if fields is not None:
                st = State(**{f: (getattr(st, f) if f in fields else None) for f in STATE_FIELDS})
            for f in STATE_FIELDS:
                a = getattr(st, f)
                if a is not None and (a.shape[0] < caps[i] or not a.flags.c_contiguous):
                    raise ValueError(f"download_many: {f} must be C-contiguous with {caps[i]} rows")
            sts.append(st)
        cs = (NvHostState * max(len(sts), 1))(*[st.to_c() for st in sts])
        sy = (C.c_int32 * max(len(systems), 1))(*systems)
        cp = (C.c_int32 * max(len(caps), 1))(*caps)
        _check(lib().nv_download_many(self.h, len(sts), sy, cs, cp))
        return [st.trimmed(cs[i].pcount) for i, st in enumerate(sts)]

    def set_clock(self, sys: int, t: float, itime: int):
        _check(lib().nv_set_clock(self.h, int(sys), float(t), int(itime)))

    def counters(self, sys: int = 0) -> NvCounters:
        c = NvCounters()
        _check(lib().nv_counters_get(self.h, int(sys), C.byref(c)))
        return c

    def events(self, sys: int = 0) -> List[tuple]:
        n = C.c_int32()
        _check(lib().nv_events_get(self.h, int(sys), None, 1 << 30, C.byref(n)))
        buf = (NvEvent * max(n.value, 1))()
        _check(lib().nv_events_get(self.h, int(sys), buf, n.value, C.byref(n)))
        return [(e.itime, e.kind, e.i, e.j) for e in buf[: n.value]]

    # ---- stages ------------------------------------------------------------------------
    def stage(self, name: str):
        if name not in STAGES:
            raise ValueError(name)
        _check(getattr(lib(), "nv_" + name)(self.h))

    def step(self, n: int = 1):
        _check(lib().nv_step(self.h, int(n)))

    def calc_velocity(self, sys: int = 0) -> np.ndarray:
        u = np.zeros((self.capacity[sys], 3), np.float64)
        _check(lib().nv_calc_velocity(self.h, int(sys), u.ctypes.data_as(C.POINTER(C.c_double))))
        return u[: self.counters(sys).pcount].copy()

    def calc_velocity_direct_at(self, sys: int, targets) -> np.ndarray:
        """FP64 direct-sum (BS) velocity at the listed 1-based slots of system sys."""
        tg = np.ascontiguousarray(np.asarray(targets, dtype=np.int32))
        u = np.zeros((tg.shape[0], 3), np.float64)
        _check(lib().nv_calc_velocity_direct_at(self.h, int(sys), tg.ctypes.data_as(C.POINTER(C.c_int32)),
                                                tg.shape[0], u.ctypes.data_as(C.POINTER(C.c_double))))
        return u

    def upload_full(self, sys: int, st: State):
        """upload plus u_sup, u_mf, curv and stretch."""
        c = st.to_full_c()
        _check(lib().nv_upload_full(self.h, int(sys), C.byref(c)))

    def download_full(self, sys: int = 0) -> State:
        """Every kept field of f(:), u_sup/u_mf/curv/stretch included."""
        cap = self.capacity[sys]
        st = State.empty_full(cap)
        c = st.to_full_c()
        _check(lib().nv_download_full(self.h, int(sys), C.byref(c), cap))
        return st.trimmed(c.pcount)

    def set_normal_fluid_noise(self, sys: int, noise):
        """noisey_xflow samples (one per step, wrapping)."""
        a = np.ascontiguousarray(np.asarray(noise, dtype=np.float64))
        _check(lib().nv_set_normal_fluid_noise(self.h, int(sys), a.ctypes.data_as(C.POINTER(C.c_double)), a.size))

    def set_normal_fluid_grid(self, sys: int, u, yp=None):
        """laizetDNS / turbDNS grid: u of shape (3, nz, ny, nx) (the file's order), yp for laizetDNS."""
        a = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
        _, nz, ny, nx = a.shape
        y = None if yp is None else np.ascontiguousarray(np.asarray(yp, dtype=np.float64))
        _check(lib().nv_set_normal_fluid_grid(self.h, int(sys), a.ctypes.data_as(C.POINTER(C.c_double)), nx, ny, nz,
                                              None if y is None else y.ctypes.data_as(C.POINTER(C.c_double))))

    def calculate_diagnostics(self):
        """calculate_diagnostics (src/diagnostic.f90:9-74) for every system, on the device."""
        _check(lib().nv_calculate_diagnostics(self.h))

    def ts_row(self, sys: int = 0) -> NvTsRow:
        row = NvTsRow()
        _check(lib().nv_ts_row_get(self.h, int(sys), C.byref(row)))
        return row

    def write_snapshot(self, sys: int, path: str):
        _check(lib().nv_write_snapshot(self.h, int(sys), path.encode()))

    def write_dump(self, sys: int, path: str):
        _check(lib().nv_write_dump(self.h, int(sys), path.encode()))

    def restore_dump(self, sys: int, path: str):
        _check(lib().nv_restore_dump(self.h, int(sys), path.encode()))

    def diagnostics(self, sys: int = 0) -> list:
        out = (C.c_int64 * 12)()
        _check(lib().nv_diagnostics(self.h, int(sys), out, 12))
        return list(out)

    def stage_times(self) -> dict:
        ms = (C.c_double * len(STAGE_TIMES))()
        _check(lib().nv_stage_times(self.h, ms, len(STAGE_TIMES)))
        return dict(zip(STAGE_TIMES, list(ms)))

    def set_near_factor(self, factor: float):
        _check(lib().nv_set_near_factor(self.h, float(factor)))

    def set_fp32_guards(self, angle: float, line: float, end: float):
        """Thresholds below which a far mixed-precision term is evaluated in FP64."""
        _check(lib().nv_set_fp32_guards(self.h, float(angle), float(line), float(end)))

    def set_root_band(self, scale: float):
        """Scale of the root-centre estimate's error bound (huge: every root test exact)."""
        _check(lib().nv_set_root_band(self.h, float(scale)))

    def set_walk_parts(self, parts: int):
        """Split of the tree walks' work (mixed: central image over groups of root children;
        FP64: unshifted / shifted images on two threads per target); 0: automatic."""
        _check(lib().nv_set_walk_parts(self.h, int(parts)))

    def set_walk_range(self, sys: int, lo: int, hi: int):
        """Tree walks compute only walk positions lo <= q < hi of system sys (one tangle split
        over GPUs); (1, capacity + 1) restores all."""
        _check(lib().nv_set_walk_range(self.h, int(sys), int(lo), int(hi)))

    def velocity_pack(self, sys: int, lo: int, count: int, dev_ptr: int):
        """Velocities of walk positions lo .. lo+count-1 into a device buffer [count][3] (a
        CUDA pointer, e.g. a torch tensor's data_ptr())."""
        _check(lib().nv_velocity_pack(self.h, int(sys), int(lo), int(count), C.c_void_p(int(dev_ptr))))

    def velocity_unpack(self, sys: int, lo: int, count: int, dev_ptr: int):
        _check(lib().nv_velocity_unpack(self.h, int(sys), int(lo), int(count), C.c_void_p(int(dev_ptr))))

    def step_velocity(self):
        """The first half of a step: up to and including the velocity pass."""
        _check(lib().nv_step_velocity(self.h))

    def step_finish(self):
        """The second half: AB3 update, topology, wrap, clock."""
        _check(lib().nv_step_finish(self.h))

    def set_event_margins(self, on: bool = True):
        """Switch the event-margin record on (and reset it) or off."""
        _check(lib().nv_set_event_margins(self.h, int(bool(on))))

    def event_margins(self, sys: int = 0) -> dict:
        """Smallest relative margins of the topology tests since set_event_margins(True)."""
        out = (C.c_double * 4)()
        _check(lib().nv_event_margins_get(self.h, int(sys), out))
        return dict(zip(("insert", "remove", "recon_distance", "recon_dot"), list(out)))

    def set_direct_split(self, targets_per_block: int):
        """Plain FP64 direct sum: 64 = one thread per target; 1, 2, 4, 8 = that many targets per
        block, terms computed by many threads and added in the reference order; 0 = automatic."""
        _check(lib().nv_set_direct_split(self.h, int(targets_per_block)))

    def set_pclose_method(self, method: int):
        """pclose of tree-less systems: 0 = cell list (default), 1 = scan every slot."""
        _check(lib().nv_set_pclose_method(self.h, int(method)))

    def set_insert_iterations(self, n: int):
        """Fixed-point rounds of the parallel pinsert (0: the serial sweep every step)."""
        _check(lib().nv_set_insert_iterations(self.h, int(n)))

    def set_timing(self, on: bool):
        _check(lib().nv_set_timing(self.h, int(bool(on))))

    def step_launches(self) -> int:
        n = C.c_int32()
        _check(lib().nv_step_launches(self.h, C.byref(n)))
        return n.value

    def sync(self):
        _check(lib().nv_sync(self.h))

    def tree_dump(self, sys: int = 0) -> np.ndarray:
        n = C.c_int32()
        _check(lib().nv_tree_dump(self.h, int(sys), None, 0, C.byref(n)))
        buf = (NvTreeNode * max(n.value, 1))()
        _check(lib().nv_tree_dump(self.h, int(sys), buf, n.value, C.byref(n)))
        return tree_nodes_to_numpy(buf, n.value)
