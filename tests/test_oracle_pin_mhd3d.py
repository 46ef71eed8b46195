"""Pin the 3D restatement (oracle/mhd3d_oracle.hpp) to the reference
mhd3d_resistive_hlld_ct.cpp compiled in place: bit-identical stage, RK2 step,
dt and main-loop steps on seeded cases (periodic / outflow / mixed
boundaries, the ideal-gas mapping and the full hybrid EOS across rho_nuc and
rho_bounce, resistive and ideal)."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_mhd3d import CASES3, make_case3

pytestmark = pytest.mark.skipif(O.ref("mhd3d") is None, reason="compiled reference (oracle/_ref) not available")


def _setup(name):
    p, s = make_case3(name)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    dt = O.ref("mhd3d").ref_mhd3d_compute_dt(C.byref(cp), O.pp(S))
    return p, cp, S, dt


@pytest.mark.parametrize("name", sorted(CASES3))
def test_compute_dt_bitwise(name):
    p, cp, S, dt = _setup(name)
    assert O.oracle().or_mhd3d_compute_dt(C.byref(cp), O.pp(S)) == dt


@pytest.mark.parametrize("name", sorted(CASES3))
def test_advance_stage_bitwise(name):
    p, cp, S, dt = _setup(name)
    a = [np.zeros_like(x) for x in S]
    b = [np.zeros_like(x) for x in S]
    O.ref("mhd3d").ref_mhd3d_advance_stage(C.byref(cp), O.pp(S), O.pp(a), dt)
    O.oracle().or_mhd3d_advance_stage(C.byref(cp), O.pp(S), O.pp(b), dt)
    for k, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"field {k}: max |d| {np.max(np.abs(x - y))}"


@pytest.mark.parametrize("name", sorted(CASES3))
def test_rk2_step_bitwise(name):
    p, cp, S, dt = _setup(name)
    a = O.m3_rk2_ref(cp, S, dt)
    b = O.m3_rk2_oracle(cp, S, dt)
    for k, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"field {k}: max |d| {np.max(np.abs(x - y))}"


@pytest.mark.parametrize("name", ["periodic_ideal", "mixed_hybrid"])
def test_main_loop_bitwise(name):
    p, cp, S, dt = _setup(name)
    cp.t_end = 10.0
    a = O.copy_state(S)
    t = C.c_double(0.0)
    O.ref("mhd3d").ref_mhd3d_main_loop(C.byref(cp), O.pp(a), 3, C.byref(t))
    b, tb = O.m3_main_loop_oracle(cp, S, 3)
    assert t.value == tb
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert O.ref("mhd3d").ref_mhd3d_divB_max(C.byref(cp), O.pp(a)) == O.oracle().or_mhd3d_divB_max(C.byref(cp), O.pp(b))
