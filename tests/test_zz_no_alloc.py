"""nv_calc_velocity_bs_static: the direct-sum velocity pass that allocates nothing.

It serves callers that keep the filament state in device memory they own and cannot let a
library allocate behind them (their own pool or budget, or no room for the synchronisation
cudaMalloc implies).  It must give the same velocities as nv_calc_velocity on the same state
(same kernels: tolerance 1e-12 relative, as for the plain path) and as the CPU oracle, on
consecutive calls that reuse its static scratch (including a smaller system after a larger
one, whose leftovers stay in the scratch), must leave its output unwritten when it rejects
the input, and must refuse systems larger than its scratch.

This file is collected last, so that a run stopping at the first failure has already run
every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import config0_params, rel_err, tangle

pytestmark = pytest.mark.gpu


def _entry():
    from nuvort_b200.abi import NvParams
    from nuvort_b200.api import lib
    L = lib()
    f = L.nv_calc_velocity_bs_static
    f.argtypes = [C.POINTER(NvParams), C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                  C.c_void_p]
    return L, f


def _static_call(p, st, t=0.0, fill=float("nan")):
    """(status, velocities) of one call on device copies of st; the output buffer starts as `fill`."""
    import torch
    L, f = _entry()
    x = torch.tensor(st.x, dtype=torch.float64, device="cuda").contiguous()
    inf = torch.tensor(st.infront, dtype=torch.int32, device="cuda")
    beh = torch.tensor(st.behind, dtype=torch.int32, device="cuda")
    u = torch.full((st.pcount, 3), fill, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = f(C.byref(p), st.pcount, x.data_ptr(), inf.data_ptr(), beh.data_ptr(), t, u.data_ptr(), None)
    torch.cuda.synchronize()
    return rc, u.cpu().numpy(), L.nv_last_error().decode()


def _static_velocity(p, st, t=0.0):
    rc, u, msg = _static_call(p, st, t)
    assert rc == 0, msg
    return u


def _handle_velocity(p, st):
    from nuvort_b200.api import Handle
    with Handle(p, [st.pcount + 16], states=[st]) as h:
        return h.calc_velocity()


def _oracle_velocity(p, st):
    from oracle import Oracle
    return Oracle(p, st).calc_velocity()


def _holed(st):
    """Two empty slots closed over by their neighbours."""
    st.infront[[9, 10]] = 0
    st.behind[[9, 10]] = 0
    st.x[[9, 10]] = 0
    st.infront[8] = 12
    st.behind[11] = 9
    return st


def _cases():
    return [(_holed(tangle(9, 0.002, n_points=3000)),
             config0_params(alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.0, 0.2, 0.5))),
            (tangle(0, 0.002, n_rings=8), config0_params())]


def test_static_entry_matches_calc_velocity_and_oracle_on_consecutive_calls():
    # the larger system first: the second, smaller call runs on a scratch array that still
    # holds the first call's slots beyond its own pcount
    for st, p in _cases():
        us = _static_velocity(p, st)
        uh = _handle_velocity(p, st)
        uo = _oracle_velocity(p, st)
        live = st.infront > 0
        assert np.all(us[~live] == 0)
        assert rel_err(us[live], uh[live]).max() <= 1e-12
        assert rel_err(us[live], uo[live]).max() <= 1e-12


def test_static_entry_same_result_twice_in_a_row():
    st, p = _cases()[1]
    a = _static_velocity(p, st)
    b = _static_velocity(p, st)
    assert np.array_equal(a, b)


def test_static_entry_rejected_links_leave_output_unwritten():
    from nuvort_b200.abi import NV_ERR_ARG
    st, p = _cases()[1]
    good = _static_velocity(p, st)  # fills the scratch with valid velocities of this system
    bad = tangle(0, 0.002, n_rings=8)
    bad.infront[4] = bad.pcount + 7
    rc, u, msg = _static_call(p, bad, fill=-123.0)
    assert rc == NV_ERR_ARG and "out of range" in msg
    assert np.all(u == -123.0)  # neither stale nor partial velocities
    bad = tangle(0, 0.002, n_rings=8)
    bad.behind[4] = 0  # live slot with an empty link on one side only
    rc, u, msg = _static_call(p, bad, fill=-123.0)
    assert rc == NV_ERR_ARG and np.all(u == -123.0)
    assert np.array_equal(_static_velocity(p, st), good)  # the entry point is usable afterwards


def test_static_entry_single_empty_slot():
    from nuvort_b200.abi import State
    z = np.zeros((1, 3))
    st = State(x=z.copy(), infront=np.zeros(1, np.int32), behind=np.zeros(1, np.int32))
    u = _static_velocity(config0_params(), st)
    assert np.array_equal(u, np.zeros((1, 3)))


def test_static_entry_refuses_oversized_systems():
    from nuvort_b200.abi import NV_ERR_CAPACITY
    L, f = _entry()
    p = config0_params()
    rc = f(C.byref(p), 32769, 1, 1, 1, 0.0, 1, None)  # refused before any pointer is used
    assert rc == NV_ERR_CAPACITY
    assert b"32768" in L.nv_last_error()


def test_static_entry_refuses_solid_walls():
    # pinned records are not among its arguments: a system with a solid wall is refused
    # before any pointer is used, and the output stays unwritten
    from nuvort_b200.abi import NV_ERR_UNSUPPORTED
    st = tangle(0, 0.002, n_rings=4)
    rc, u, msg = _static_call(config0_params(boundary_y="solid"), st, fill=-7.0)
    assert rc == NV_ERR_UNSUPPORTED and "solid" in msg
    assert np.all(u == -7.0)
