"""nv_calc_velocity_bs_static: the direct-sum velocity pass that allocates nothing.

It serves callers that keep the filament state in device memory they own and cannot let a
library allocate behind them (their own pool or budget, or no room for the synchronisation
cudaMalloc implies).  It must give the same velocities as nv_calc_velocity on the same state
(same kernels: tolerance 1e-12 relative, as for the plain path), on consecutive calls that
reuse its static scratch, and must refuse systems larger than its scratch.
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


def _static_velocity(p, st, t=0.0):
    import torch
    L, f = _entry()
    x = torch.tensor(st.x, dtype=torch.float64, device="cuda").contiguous()
    inf = torch.tensor(st.infront, dtype=torch.int32, device="cuda")
    beh = torch.tensor(st.behind, dtype=torch.int32, device="cuda")
    u = torch.full((st.pcount, 3), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = f(C.byref(p), st.pcount, x.data_ptr(), inf.data_ptr(), beh.data_ptr(), t, u.data_ptr(), None)
    assert rc == 0, L.nv_last_error().decode()
    return u.cpu().numpy()


def _handle_velocity(p, st):
    from nuvort_b200.api import Handle
    with Handle(p, [st.pcount + 16], states=[st]) as h:
        return h.calc_velocity()


def test_static_entry_matches_calc_velocity_on_consecutive_calls():
    cases = [(tangle(0, 0.002, n_rings=8), config0_params()),
             (tangle(9, 0.002, n_points=3000),
              config0_params(alpha=(0.1, 0.01), normal_velocity="uniform", norm_vel_vec=(0.0, 0.2, 0.5)))]
    # hole in the second system: two empty slots closed over by their neighbours
    st2 = cases[1][0]
    st2.infront[[9, 10]] = 0
    st2.behind[[9, 10]] = 0
    st2.x[[9, 10]] = 0
    st2.infront[8] = 12
    st2.behind[11] = 9
    for st, p in cases:  # two calls in a row through the same static scratch
        us = _static_velocity(p, st)
        uh = _handle_velocity(p, st)
        live = st.infront > 0
        assert np.all(us[~live] == 0)
        assert rel_err(us[live], uh[live]).max() <= 1e-12


def test_static_entry_refuses_oversized_systems():
    from nuvort_b200.abi import NV_ERR_CAPACITY
    L, f = _entry()
    p = config0_params()
    rc = f(C.byref(p), 32769, 1, 1, 1, 0.0, 1, None)  # refused before any pointer is used
    assert rc == NV_ERR_CAPACITY
    assert b"32768" in L.nv_last_error()
