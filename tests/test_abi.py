"""Host-side checks of the C ABI: the library loads, exports every declared entry point,
and its host-only functions (defaults, parameter checks, the run.in reader) behave like the
reference's (src/cdata.f90:76-241, src/initial.f90:14-180).  No CUDA call is made here."""
import ctypes as C
import os
import re

import pytest

from nuvort_b200 import api
from nuvort_b200.abi import (NV_BC_OPEN, NV_BC_PERIODIC, NV_ERR_TIMESTEP, NV_ERR_UNSUPPORTED,
                             NV_NF_UNIFORM, NV_NF_XFLOW, NV_PREC_MIXED, NV_VEL_BS, NV_VEL_TREE,
                             NvParams, default_params, make_params)

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*|void)\s*\**\s*(nv_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = api.lib()
    names = declared("nuvort_gpu.h")
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_exports_every_declared_symbol():
    import oracle
    text = open(os.path.join(ROOT, "oracle", "nuvort_oracle.h")).read()
    names = re.findall(r"^\s*(?:int|void|int32_t|const char \*)\s*(or_\w+)\s*\(", text, re.M)
    lib = oracle.lib()
    assert names and all(hasattr(lib, n) for n in names)


def test_defaults_match_python_mirror():
    p = NvParams()
    assert api.lib().nv_params_default(C.byref(p)) == 0
    q = default_params()
    assert bytes(p) == bytes(q)


def test_timestep_check():
    ok = make_params(dt=2e-5, delta=0.002, box_size=0.1)
    api.check_params(ok)
    bad = make_params(dt=2e-4, delta=0.002, box_size=0.1)
    with pytest.raises(api.NuvortError) as e:
        api.check_params(bad)
    assert e.value.code == NV_ERR_TIMESTEP
    bad.overide_timestep_check = 1
    api.check_params(bad)


def test_unsupported_options_are_refused():
    p = make_params(dt=2e-5, delta=0.002, box_size=0.1, boundary_x="solid")
    api.check_params(p)  # solid walls run in FP64
    p = make_params(dt=2e-5, delta=0.002, box_size=0.1, boundary_x="solid", precision="mixed")
    with pytest.raises(api.NuvortError) as e:
        api.check_params(p)
    assert e.value.code == NV_ERR_UNSUPPORTED
    p = make_params(dt=2e-5, delta=0.002, box_size=0.1, velocity="Tree", tree_theta=0.4, boundary_z="open")
    with pytest.raises(api.NuvortError):
        api.check_params(p)


def test_run_in_reader(tmp_path):
    f = tmp_path / "run.in"
    f.write_text("nsteps 200\nshots 10\ndt 2E-5\ndelta 0.002\nbox_size 0.1 0.1 0.1\n"
                 "velocity Tree\ntree_theta 0.4\nboundary_z open\nnormal_velocity xflow\n"
                 "norm_vel_xflow 1d0\nalpha 0.1 0.01\nunknown_key 5\nquant_circ 9.97E-4\n"
                 "precision mixed\n")
    p = api.read_run_file(str(f))
    assert p.nsteps == 200 and p.shots == 10 and p.dt == 2e-5 and p.delta == 0.002
    assert list(p.box_size) == [0.1, 0.1, 0.1]
    assert p.velocity == NV_VEL_TREE and p.tree_theta == 0.4
    assert list(p.boundary) == [NV_BC_PERIODIC, NV_BC_PERIODIC, NV_BC_OPEN]
    assert p.normal_velocity == NV_NF_XFLOW and p.norm_vel_xflow == 1.0
    assert list(p.alpha) == [0.1, 0.01] and p.precision == NV_PREC_MIXED


def test_run_in_malformed_value_ends_the_read(tmp_path):
    # src/cdata.f90:145-157: the value's iostat is the loop condition, so a list with too
    # few items (box_size with one number) stops the read after assigning what it read.
    f = tmp_path / "run.in"
    f.write_text("nsteps 100000\nshots 10\ndt 1E-4\ndelta 0.005\nbox_size 0.4\nvelocity LIA\n")
    p = api.read_run_file(str(f))
    assert p.nsteps == 100000 and p.delta == 0.005
    assert list(p.box_size) == [0.4, 0.0, 0.0]
    assert p.velocity == NV_VEL_BS  # never read: default kept


def test_run_in_uniform_extension(tmp_path):
    f = tmp_path / "run.in"
    f.write_text("normal_velocity uniform\nnorm_vel_vec 0 0 0.5\n")
    p = api.read_run_file(str(f))
    assert p.normal_velocity == NV_NF_UNIFORM and list(p.norm_vel_vec) == [0.0, 0.0, 0.5]


def test_run_in_normal_fluid_fields(tmp_path):
    from nuvort_b200.abi import NV_NF_SHEAR_XFLOW, NV_NF_TURB_DNS
    from nuvort_b200.api import read_run_file
    f = tmp_path / "run.in"
    f.write_text("normal_velocity shear_xflow\nnorm_shear_omega 3.5\nnoise_file noise/wn_snr_25.log\n"
                 "norm_vel_xflow 0.25\n")
    p = read_run_file(str(f))
    assert p.normal_velocity == NV_NF_SHEAR_XFLOW and p.norm_shear_omega == 3.5 and p.norm_vel_xflow == 0.25
    f.write_text("normal_velocity turbDNS\n")
    assert read_run_file(str(f)).normal_velocity == NV_NF_TURB_DNS
