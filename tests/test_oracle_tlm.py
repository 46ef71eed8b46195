"""CPU checks of the oracle's dual-number tangent-linear build of the 2D MHD
step (or_mhd2d_tlm): its value part is bitwise the double restatement (which
is pinned to the compiled reference), and its tangent J v equals central
finite differences of the restatement with the same dt sequence."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_adjoint import make_case_adj as _case


def _step_oracle(p, S, dts):
    cp = p.to_c()
    S = [a.copy() for a in S]
    for dt in dts:
        if p.gravity_on:
            gx, gy, _, _ = O.m2_gravity_oracle(cp, S[0], mode=3)
        else:
            gx = gy = np.zeros(p.Nx * p.Ny)
        S = O.m2_rk2_oracle(cp, S, gx, gy, dt, mode=3)
    return S


@pytest.mark.parametrize("periodic,grav", [(False, True), (True, False)])
def test_tlm_values_bitwise_and_tangent_matches_fd(periodic, grav):
    p, U, B = _case(periodic, grav, nx=10, ny=8)
    S0 = O.state_list(U, B)
    cp = p.to_c()
    dts = np.array([O.oracle().or_mhd2d_compute_dt(C.byref(cp), O.pp(S0))] * 2)
    rng = np.random.default_rng(2)
    V = [rng.normal(size=a.size) * (np.abs(a).mean() + 1e-3) for a in S0]
    vals, tans = O.copy_state(S0), O.copy_state(V)
    assert O.oracle().or_mhd2d_tlm(C.byref(cp), O.pp(vals), O.pp(tans), len(dts), O.dp(dts)) == 0
    ref = _step_oracle(p, S0, dts)
    for a, b in zip(vals, ref):
        assert np.array_equal(a, b)
    h = 1e-7
    Sp = _step_oracle(p, [a + h * v for a, v in zip(S0, V)], dts)
    Sm = _step_oracle(p, [a - h * v for a, v in zip(S0, V)], dts)
    for k, (t, a, b) in enumerate(zip(tans, Sp, Sm)):
        fd = (a - b) / (2 * h)
        assert np.max(np.abs(t - fd)) <= 1e-6 * (np.max(np.abs(fd)) + 1e-12), f"field {k}"
