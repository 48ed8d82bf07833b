"""ctypes mirror of include/nuvort_gpu.h (records and constants).

The parameter record carries the reference's run.in keys (src/cdata.f90:131-241); the
state record carries the fields of ``type(qvort)`` (src/cdata.f90:19-29) that the hot path
touches.  Both the GPU library binding (:mod:`nuvort_b200.api`) and the test-only CPU
oracle binding use these records, so both sides receive byte-identical inputs.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

# status codes
NV_OK = 0
NV_ERR_ARG = -1
NV_ERR_CUDA = -2
NV_ERR_CAPACITY = -3
NV_ERR_SINGULAR = -4
NV_ERR_TREE_DEPTH = -5
NV_ERR_NAN = -6
NV_ERR_EMPTY = -7
NV_ERR_TIMESTEP = -8
NV_ERR_UNSUPPORTED = -9
NV_ERR_STATE = -10
NV_ERR_QUEUE = -11
NV_ERR_IO = -12
NV_ERR_TIMEOUT = -13

ERR_NAMES = {v: k for k, v in globals().items() if k.startswith("NV_ERR_") or k == "NV_OK"}

NV_VEL_LIA, NV_VEL_BS, NV_VEL_TREE = 0, 1, 2
NV_BC_PERIODIC, NV_BC_OPEN, NV_BC_SOLID = 0, 1, 2
NV_NF_ZERO, NV_NF_XFLOW, NV_NF_UNIFORM = 0, 1, 2
NV_NF_SHEAR_XFLOW, NV_NF_CHANNEL, NV_NF_YCHANNEL, NV_NF_NOISEY_XFLOW = 3, 4, 5, 6
NV_NF_LAIZET_DNS, NV_NF_TURB_DNS = 7, 8
NV_PREC_FP64, NV_PREC_MIXED = 0, 1
NV_EV_INSERT, NV_EV_RECON, NV_EV_REMOVE, NV_EV_LOOPKILL, NV_EV_WALL, NV_EV_CLEAR = 1, 2, 3, 4, 5, 6
# events whose j is a count of points, not a slot
EV_COUNT_KINDS = (NV_EV_LOOPKILL, NV_EV_WALL, NV_EV_CLEAR)
NV_TREE_MAX_DEPTH = 42

VELOCITY = {"LIA": NV_VEL_LIA, "BS": NV_VEL_BS, "Tree": NV_VEL_TREE}
BOUNDARY = {"periodic": NV_BC_PERIODIC, "open": NV_BC_OPEN, "solid": NV_BC_SOLID}
NORMAL = {"zero": NV_NF_ZERO, "xflow": NV_NF_XFLOW, "uniform": NV_NF_UNIFORM, "shear_xflow": NV_NF_SHEAR_XFLOW,
          "channel": NV_NF_CHANNEL, "ychannel": NV_NF_YCHANNEL, "noisey_xflow": NV_NF_NOISEY_XFLOW,
          "laizetDNS": NV_NF_LAIZET_DNS, "turbDNS": NV_NF_TURB_DNS}


class NvParams(C.Structure):
    _fields_ = [
        ("nsteps", C.c_int32),
        ("shots", C.c_int32),
        ("recon_shots", C.c_int32),
        ("velocity", C.c_int32),
        ("boundary", C.c_int32 * 3),
        ("normal_velocity", C.c_int32),
        ("tree_extra_correction", C.c_int32),
        ("nan_test", C.c_int32),
        ("overide_timestep_check", C.c_int32),
        ("precision", C.c_int32),
        ("dt", C.c_double),
        ("delta", C.c_double),
        ("quant_circ", C.c_double),
        ("corea", C.c_double),
        ("box_size", C.c_double * 3),
        ("tree_theta", C.c_double),
        ("norm_vel_xflow", C.c_double),
        ("norm_vel_vec", C.c_double * 3),
        ("alpha", C.c_double * 2),
        ("super_velocity", C.c_double * 3),
        ("normal_fluid_cutoff", C.c_double),
        ("t_zero_normal_fluid", C.c_double),
        ("norm_shear_omega", C.c_double),
    ]


class NvHostState(C.Structure):
    _fields_ = [
        ("pcount", C.c_int32),
        ("x", C.POINTER(C.c_double)),
        ("u", C.POINTER(C.c_double)),
        ("u1", C.POINTER(C.c_double)),
        ("u2", C.POINTER(C.c_double)),
        ("ghosti", C.POINTER(C.c_double)),
        ("ghostb", C.POINTER(C.c_double)),
        ("infront", C.POINTER(C.c_int32)),
        ("behind", C.POINTER(C.c_int32)),
        ("closest", C.POINTER(C.c_int32)),
        ("closestd", C.POINTER(C.c_double)),
        ("wpinned", C.POINTER(C.c_int32)),
        ("pinnedi", C.POINTER(C.c_int32)),
        ("pinnedb", C.POINTER(C.c_int32)),
    ]


class NvFullState(C.Structure):
    """nv_full_state: every kept field of type(qvort) (file I/O)."""
    _fields_ = [
        ("pcount", C.c_int32),
        ("x", C.POINTER(C.c_double)),
        ("u", C.POINTER(C.c_double)),
        ("u1", C.POINTER(C.c_double)),
        ("u2", C.POINTER(C.c_double)),
        ("u_mf", C.POINTER(C.c_double)),
        ("u_sup", C.POINTER(C.c_double)),
        ("curv", C.POINTER(C.c_double)),
        ("stretch", C.POINTER(C.c_double)),
        ("ghosti", C.POINTER(C.c_double)),
        ("ghostb", C.POINTER(C.c_double)),
        ("infront", C.POINTER(C.c_int32)),
        ("behind", C.POINTER(C.c_int32)),
        ("closest", C.POINTER(C.c_int32)),
        ("closestd", C.POINTER(C.c_double)),
        ("wpinned", C.POINTER(C.c_int32)),
        ("pinnedi", C.POINTER(C.c_int32)),
        ("pinnedb", C.POINTER(C.c_int32)),
    ]


class NvTsRow(C.Structure):
    """nv_ts_row: one data/ts.log row (print_info) and the values behind it."""
    _fields_ = [
        ("itime", C.c_int32),
        ("live", C.c_int32),
        ("recon_count", C.c_int32),
        ("wall_recon_count", C.c_int32),
        ("remove_count", C.c_int32),
        ("reserved", C.c_int32),
        ("tree_eval", C.c_int64),
        ("t", C.c_double),
        ("delta", C.c_double),
        ("avg_sep", C.c_double),
        ("total_length", C.c_double),
        ("maxu", C.c_double),
        ("maxdu", C.c_double),
        ("mean_u_sup", C.c_double),
        ("mean_u_mf", C.c_double),
        ("kappa_bar", C.c_double),
        ("kappa_min", C.c_double),
        ("kappa_max", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}


class NvEvent(C.Structure):
    _fields_ = [("itime", C.c_int32), ("kind", C.c_int32), ("i", C.c_int32), ("j", C.c_int32)]


class NvCounters(C.Structure):
    _fields_ = [
        ("pcount", C.c_int32),
        ("live", C.c_int32),
        ("recon_count", C.c_int32),
        ("remove_count", C.c_int32),
        ("insert_count", C.c_int32),
        ("loop_kills", C.c_int32),
        ("tree_eval", C.c_int64),
        ("tree_tests", C.c_int64),
        ("itime", C.c_int32),
        ("n_events", C.c_int32),
        ("t", C.c_double),
        ("event_hash", C.c_uint64),
        ("wall_recon_count", C.c_int32),
        ("reserved", C.c_int32),
    ]


class NvTreeNode(C.Structure):
    """One octree node in preorder (the oracle's or_tree_node / the library's nv_tree_node)."""
    _fields_ = [
        ("pos", C.c_double * 3),
        ("width", C.c_double),
        ("cent", C.c_double * 3),
        ("circ", C.c_double * 3),
        ("pcount", C.c_int32),
        ("depth", C.c_int32),
        ("leaf", C.c_int32),
        ("first_next", C.c_int32),
    ]


def default_params() -> NvParams:
    """Reference defaults, src/cdata.f90:76-127 (same values as nv_params_default)."""
    p = NvParams()
    p.nsteps = 0
    p.shots = 1
    p.recon_shots = 1
    p.velocity = NV_VEL_BS
    for k in range(3):
        p.boundary[k] = NV_BC_PERIODIC
    p.normal_velocity = NV_NF_ZERO
    p.tree_extra_correction = 1
    p.nan_test = 1
    p.overide_timestep_check = 0
    p.precision = NV_PREC_FP64
    p.dt = 0.0
    p.delta = 0.0
    p.quant_circ = 9.97e-4
    p.corea = 8.244023e-9
    p.tree_theta = 0.0
    p.norm_vel_xflow = 0.5
    p.normal_fluid_cutoff = 1e8
    p.t_zero_normal_fluid = 1e8
    p.norm_shear_omega = 0.0
    return p


def make_params(**kw) -> NvParams:
    """Build an NvParams from run.in-style keyword values (strings or numbers)."""
    p = default_params()
    for key, val in kw.items():
        if key == "velocity":
            p.velocity = VELOCITY[val] if isinstance(val, str) else int(val)
        elif key in ("boundary_x", "boundary_y", "boundary_z"):
            p.boundary["xyz".index(key[-1])] = BOUNDARY[val] if isinstance(val, str) else int(val)
        elif key == "boundary":
            for k in range(3):
                p.boundary[k] = BOUNDARY[val] if isinstance(val, str) else int(val)
        elif key == "normal_velocity":
            p.normal_velocity = NORMAL[val] if isinstance(val, str) else int(val)
        elif key == "precision":
            p.precision = {"fp64": NV_PREC_FP64, "mixed": NV_PREC_MIXED}[val] if isinstance(val, str) else int(val)
        elif key in ("box_size", "norm_vel_vec", "super_velocity", "alpha"):
            arr = getattr(p, key)
            vals = [val] * len(arr) if np.isscalar(val) else list(val)
            for k, v in enumerate(vals):
                arr[k] = float(v)
        elif key in ("tree_extra_correction", "nan_test", "overide_timestep_check"):
            setattr(p, key, int(bool(val)))
        elif key in ("nsteps", "shots", "recon_shots"):
            setattr(p, key, int(val))
        else:
            if not hasattr(p, key):
                raise KeyError(f"unknown parameter {key!r}")
            setattr(p, key, float(val))
    return p


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return C.POINTER(C.c_double)()
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: Optional[np.ndarray]):
    if a is None:
        return C.POINTER(C.c_int32)()
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_int32))


@dataclass
class State:
    """Host copy of one system's filament state: 1-based slots stored at rows 0..pcount-1.

    ``x``, ``u``, ``u1``, ``u2``, ``ghosti``, ``ghostb`` are (n, 3) float64; ``infront``,
    ``behind``, ``closest`` are int32 (0 = empty / none); ``closestd`` float64.  Solid walls:
    ``wpinned`` (n, 3) int32 in -1/0/1, ``pinnedi``, ``pinnedb`` (n,) int32 0/1 (None: no
    pinned points).
    """
    x: np.ndarray
    infront: np.ndarray
    behind: np.ndarray
    u: Optional[np.ndarray] = None
    u1: Optional[np.ndarray] = None
    u2: Optional[np.ndarray] = None
    ghosti: Optional[np.ndarray] = None
    ghostb: Optional[np.ndarray] = None
    closest: Optional[np.ndarray] = None
    closestd: Optional[np.ndarray] = None
    # fields only the diagnostics and the files use: f(:)%u_mf, u_sup (n, 3), curv, stretch (n,)
    u_mf: Optional[np.ndarray] = None
    u_sup: Optional[np.ndarray] = None
    curv: Optional[np.ndarray] = None
    stretch: Optional[np.ndarray] = None
    wpinned: Optional[np.ndarray] = None
    pinnedi: Optional[np.ndarray] = None
    pinnedb: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def pcount(self) -> int:
        return int(self.x.shape[0])

    @staticmethod
    def empty(cap: int) -> "State":
        z3 = lambda: np.zeros((cap, 3), np.float64)
        return State(x=z3(), infront=np.zeros(cap, np.int32), behind=np.zeros(cap, np.int32),
                     u=z3(), u1=z3(), u2=z3(), ghosti=z3(), ghostb=z3(),
                     closest=np.zeros(cap, np.int32), closestd=np.zeros(cap, np.float64),
                     wpinned=np.zeros((cap, 3), np.int32), pinnedi=np.zeros(cap, np.int32),
                     pinnedb=np.zeros(cap, np.int32))

    @staticmethod
    def empty_full(cap: int) -> "State":
        st = State.empty(cap)
        st.u_mf = np.zeros((cap, 3), np.float64)
        st.u_sup = np.zeros((cap, 3), np.float64)
        st.curv = np.zeros(cap, np.float64)
        st.stretch = np.zeros(cap, np.float64)
        return st

    def copy(self) -> "State":
        cp = lambda a: None if a is None else np.array(a, copy=True)
        return State(**{f: cp(getattr(self, f)) for f in FIELDS})

    def trimmed(self, n: int) -> "State":
        cut = lambda a: None if a is None else np.ascontiguousarray(a[:n])
        return State(**{f: cut(getattr(self, f)) for f in FIELDS})

    def to_full_c(self) -> NvFullState:
        """nv_full_state over this state's arrays (float64 / int32, made contiguous)."""
        self.to_c()
        for name in ("u_mf", "u_sup", "curv", "stretch"):
            a = getattr(self, name)
            if a is not None:
                setattr(self, name, np.ascontiguousarray(a, dtype=np.float64))
        s = NvFullState()
        s.pcount = self.pcount
        for name in ("x", "u", "u1", "u2", "u_mf", "u_sup", "curv", "stretch", "ghosti", "ghostb", "closestd"):
            setattr(s, name, _dptr(getattr(self, name)))
        for name in ("infront", "behind", "closest", "wpinned", "pinnedi", "pinnedb"):
            setattr(s, name, _iptr(getattr(self, name)))
        return s

    def to_c(self) -> NvHostState:
        for name in ("x", "u", "u1", "u2", "ghosti", "ghostb", "closestd"):
            a = getattr(self, name)
            if a is not None:
                setattr(self, name, np.ascontiguousarray(a, dtype=np.float64))
        for name in ("infront", "behind", "closest", "wpinned", "pinnedi", "pinnedb"):
            a = getattr(self, name)
            if a is not None:
                setattr(self, name, np.ascontiguousarray(a, dtype=np.int32))
        s = NvHostState()
        s.pcount = self.pcount
        s.x = _dptr(self.x)
        s.u = _dptr(self.u)
        s.u1 = _dptr(self.u1)
        s.u2 = _dptr(self.u2)
        s.ghosti = _dptr(self.ghosti)
        s.ghostb = _dptr(self.ghostb)
        s.infront = _iptr(self.infront)
        s.behind = _iptr(self.behind)
        s.closest = _iptr(self.closest)
        s.closestd = _dptr(self.closestd)
        s.wpinned = _iptr(self.wpinned)
        s.pinnedi = _iptr(self.pinnedi)
        s.pinnedb = _iptr(self.pinnedb)
        return s

    @property
    def live(self) -> np.ndarray:
        return self.infront > 0


FIELDS = ("x", "infront", "behind", "u", "u1", "u2", "ghosti", "ghostb", "closest", "closestd", "u_mf", "u_sup",
          "curv", "stretch", "wpinned", "pinnedi", "pinnedb")


TREE_NODE_DTYPE = np.dtype([("pos", "<f8", 3), ("width", "<f8"), ("cent", "<f8", 3), ("circ", "<f8", 3),
                            ("pcount", "<i4"), ("depth", "<i4"), ("leaf", "<i4"), ("first_next", "<i4")])


def tree_nodes_to_numpy(buf, n: int) -> np.ndarray:
    """Copy n NvTreeNode records into a structured numpy array."""
    assert TREE_NODE_DTYPE.itemsize == C.sizeof(NvTreeNode)
    return np.frombuffer(bytes(memoryview(buf))[: n * TREE_NODE_DTYPE.itemsize], dtype=TREE_NODE_DTYPE).copy()


_M64 = (1 << 64) - 1


def _digest_mix(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def event_digest(events, seq0: int = 0) -> int:
    """Host mirror of the device event digest: the sum (mod 2^64) over events, in order,
    of a hash of (sequence number, itime, kind, i, j); events as (itime, kind, i, j) with
    system-local slots, the first one numbered seq0.  Equals nv_counters.event_hash for the
    same event sequence."""
    tot = 0
    for q, (itime, kind, i, j) in enumerate(events):
        h = _digest_mix((seq0 + q) & 0xFFFFFFFF)
        h = _digest_mix(h ^ (((i & 0xFFFFFFFF) << 32) | (j & 0xFFFFFFFF)))
        h = _digest_mix(h ^ (((itime & 0xFFFFFFFF) << 8) | (kind & 0xFFFFFFFF)))
        tot = (tot + h) & _M64
    return tot
