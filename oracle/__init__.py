"""Python binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates the reference Fortran line by line in C++ (oracle/nuvort_oracle.cpp).
Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may use
it, and only as the checker; the product library never calls it.

Parity status: unpinned (the reference has no tests or golden vectors and cannot be
compiled in this environment); see oracle/README.md.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Optional, Sequence

import numpy as np

from nuvort_b200.abi import (NvCounters, NvEvent, NvFullState, NvParams, NvTreeNode, NvTsRow, State, NV_OK,
                             ERR_NAMES, tree_nodes_to_numpy)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libnuvort_oracle.so")

_lib = None


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc only; no reference sources are used).

    make tracks the dependencies (the oracle and the shared ABI header), so this is cheap
    when the library is current; without a compiler (a box that only runs tests) a present
    library is used as is."""
    try:
        subprocess.run(["make", "-s", "-C", HERE] + (["-B"] if force else []), check=True)
    except (OSError, subprocess.CalledProcessError):
        if not os.path.exists(LIB_PATH):
            raise
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        vp = C.c_void_p
        L.or_create.argtypes = [P(NvParams), P(vp)]
        for name in ("or_destroy", "or_ghostp", "or_construct_tree", "or_pmotion", "or_pinsert",
                     "or_pclose", "or_precon", "or_wall_recon", "or_premove", "or_enforce_boundary",
                     "or_empty_tree",
                     "or_end_step"):
            getattr(L, name).argtypes = [vp]
        L.or_upload.argtypes = [vp, vp]
        L.or_download.argtypes = [vp, vp, C.c_int32]
        L.or_set_clock.argtypes = [vp, C.c_double, C.c_int32]
        L.or_counters_get.argtypes = [vp, P(NvCounters)]
        L.or_events_get.argtypes = [vp, P(NvEvent), C.c_int32, P(C.c_int32)]
        L.or_step.argtypes = [vp, C.c_int32]
        L.or_calc_velocity.argtypes = [vp, P(C.c_double)]
        L.or_calc_velocity_targets.argtypes = [vp, C.c_int32, P(C.c_int32), C.c_int32, P(C.c_double)]
        L.or_tree_dump.argtypes = [vp, P(NvTreeNode), C.c_int32, P(C.c_int32)]
        L.or_set_normal_fluid_noise.argtypes = [vp, P(C.c_double), C.c_int32]
        L.or_set_normal_fluid_grid.argtypes = [vp, P(C.c_double), C.c_int32, C.c_int32, C.c_int32, P(C.c_double)]
        L.or_calculate_diagnostics.argtypes = [vp]
        L.or_ts_row_get.argtypes = [vp, P(NvTsRow)]
        L.or_download_full.argtypes = [vp, P(NvFullState), C.c_int32]
        L.or_upload_full.argtypes = [vp, P(NvFullState)]
        L.or_write_snapshot.argtypes = [vp, C.c_char_p]
        L.or_write_dump.argtypes = [vp, C.c_char_p]
        L.or_set_event_margins.argtypes = [vp, C.c_int32]
        L.or_event_margins_get.argtypes = [vp, P(C.c_double)]
        L.or_set_threads.argtypes = [C.c_int32]
        L.or_get_threads.restype = C.c_int32
        L.or_last_error.restype = C.c_char_p
        _lib = L
    return _lib


class OracleError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def _check(rc: int):
    if rc != NV_OK:
        raise OracleError(rc, lib().or_last_error().decode())


def set_threads(n: int):
    lib().or_set_threads(int(n))


def get_threads() -> int:
    return int(lib().or_get_threads())


class Oracle:
    """One filament system on the CPU, with the reference's stage procedures."""

    def __init__(self, params: NvParams, state: Optional[State] = None, t: float = 0.0, itime: int = 0):
        self.params = params
        h = C.c_void_p()
        _check(lib().or_create(C.byref(params), C.byref(h)))
        self.h = h
        if state is not None:
            self.upload(state)
            self.set_clock(t, itime)

    def close(self):
        if self.h:
            lib().or_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload(self, st: State):
        cst = st.to_c()
        _check(lib().or_upload(self.h, C.byref(cst)))

    def download(self, cap: Optional[int] = None) -> State:
        n = self.counters().pcount
        cap = max(n, 1) if cap is None else cap
        st = State.empty(cap)
        cst = st.to_c()
        _check(lib().or_download(self.h, C.byref(cst), cap))
        return st.trimmed(cst.pcount)

    def set_clock(self, t: float, itime: int):
        _check(lib().or_set_clock(self.h, t, itime))

    def counters(self) -> NvCounters:
        c = NvCounters()
        _check(lib().or_counters_get(self.h, C.byref(c)))
        return c

    def events(self) -> List[tuple]:
        n_tot = self.counters().n_events
        buf = (NvEvent * max(n_tot, 1))()
        n = C.c_int32()
        _check(lib().or_events_get(self.h, buf, n_tot, C.byref(n)))
        return [(e.itime, e.kind, e.i, e.j) for e in buf[: n.value]]

    def stage(self, name: str):
        _check(getattr(lib(), "or_" + name)(self.h))

    def step(self, n: int = 1):
        _check(lib().or_step(self.h, int(n)))

    def calc_velocity(self) -> np.ndarray:
        n = self.counters().pcount
        u = np.zeros((n, 3), np.float64)
        _check(lib().or_calc_velocity(self.h, u.ctypes.data_as(C.POINTER(C.c_double))))
        return u

    def calc_velocity_targets(self, velocity: int, targets: Sequence[int]) -> np.ndarray:
        tg = np.ascontiguousarray(np.asarray(targets, dtype=np.int32))
        u = np.zeros((tg.shape[0], 3), np.float64)
        _check(lib().or_calc_velocity_targets(self.h, int(velocity), tg.ctypes.data_as(C.POINTER(C.c_int32)),
                                              tg.shape[0], u.ctypes.data_as(C.POINTER(C.c_double))))
        return u

    def set_normal_fluid_noise(self, noise):
        a = np.ascontiguousarray(np.asarray(noise, dtype=np.float64))
        _check(lib().or_set_normal_fluid_noise(self.h, a.ctypes.data_as(C.POINTER(C.c_double)), a.size))

    def set_normal_fluid_grid(self, u, yp=None):
        a = np.ascontiguousarray(np.asarray(u, dtype=np.float64))
        _, nz, ny, nx = a.shape
        y = None if yp is None else np.ascontiguousarray(np.asarray(yp, dtype=np.float64))
        _check(lib().or_set_normal_fluid_grid(self.h, a.ctypes.data_as(C.POINTER(C.c_double)), nx, ny, nz,
                                              None if y is None else y.ctypes.data_as(C.POINTER(C.c_double))))

    def calculate_diagnostics(self):
        _check(lib().or_calculate_diagnostics(self.h))

    def ts_row(self) -> NvTsRow:
        row = NvTsRow()
        _check(lib().or_ts_row_get(self.h, C.byref(row)))
        return row

    def download_full(self) -> State:
        n = self.counters().pcount
        st = State.empty_full(max(n, 1))
        c = st.to_full_c()
        _check(lib().or_download_full(self.h, C.byref(c), max(n, 1)))
        return st.trimmed(c.pcount)

    def upload_full(self, st: State):
        c = st.to_full_c()
        _check(lib().or_upload_full(self.h, C.byref(c)))

    def write_snapshot(self, path: str):
        _check(lib().or_write_snapshot(self.h, path.encode()))

    def write_dump(self, path: str):
        _check(lib().or_write_dump(self.h, path.encode()))

    def set_event_margins(self, on: bool = True):
        _check(lib().or_set_event_margins(self.h, int(bool(on))))

    def event_margins(self) -> dict:
        out = (C.c_double * 4)()
        _check(lib().or_event_margins_get(self.h, out))
        return dict(zip(("insert", "remove", "recon_distance", "recon_dot"), list(out)))

    def tree_dump(self) -> np.ndarray:
        n = C.c_int32()
        _check(lib().or_tree_dump(self.h, None, 0, C.byref(n)))
        buf = (NvTreeNode * max(n.value, 1))()
        _check(lib().or_tree_dump(self.h, buf, n.value, C.byref(n)))
        return tree_nodes_to_numpy(buf, n.value)
