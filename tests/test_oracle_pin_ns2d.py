"""Pin the 2D Navier-Stokes restatement (oracle/ns2d_oracle.hpp) to the
reference navier_stokes_2d_hllc_poisson.cpp compiled in place: bit-identical
compute_rhs (HLLC, viscous stress, spectral gravity) and compute_dt, the
main-loop Heun step composed from the reference's compute_rhs, and the
library's host IC against the restated one."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_ns2d import CASES_NS, make_case_ns

needs_ref = pytest.mark.skipif(O.ref("fft") is None, reason="compiled reference (oracle/_ref) not available")


@needs_ref
@pytest.mark.parametrize("name", sorted(CASES_NS))
def test_rhs_and_dt_bitwise(name):
    p, s = make_case_ns(name)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    want = O.ns_ref_rhs(cp, S)
    got = O.ns_rhs_oracle(cp, S)
    for k, (x, y) in enumerate(zip(want, got)):
        assert np.array_equal(x, y), f"component {k}"
    assert O.oracle().or_ns2d_compute_dt(C.byref(cp), O.pp(S)) == O.ns_ref_dt(cp, S)


@needs_ref
@pytest.mark.parametrize("name", ["collapse_ic", "kicked_viscous", "floors"])
def test_heun_step_bitwise(name):
    """The main() loop body (NS:759-783) composed from the reference's own
    compute_dt and compute_rhs, against the oracle's main loop, 2 steps."""
    p, s = make_case_ns(name)
    cp = p.to_c()
    U = [a.copy() for a in s.arrays()]
    t = 0.0
    for _ in range(2):
        dt = O.ns_ref_dt(cp, U)
        if t + dt > p.t_end:
            dt = p.t_end - t
        k1 = O.ns_ref_rhs(cp, U)
        U1 = [u + dt * k for u, k in zip(U, k1)]
        U1[0] = np.where(U1[0] < p.floor_rho, p.floor_rho, U1[0])
        k2 = O.ns_ref_rhs(cp, U1)
        U = [u + 0.5 * dt * (a + b) for u, a, b in zip(U, k1, k2)]
        U[0] = np.where(U[0] < p.floor_rho, p.floor_rho, U[0])
        t += dt
    got, tg = O.ns_main_loop_oracle(cp, s.arrays(), 2)
    assert tg == t
    for k, (x, y) in enumerate(zip(U, got)):
        assert np.array_equal(x, y), f"component {k}"


def test_library_ic_equals_restatement():
    """cc_ic_ns2d_collapse (host code of the library) == the oracle's
    restatement of NS:627-689 bit for bit (both draw from std::mt19937 and
    libstdc++'s normal_distribution)."""
    from core_collapse_b200.ns2d import ParamsNS, ic_collapse
    for kw in (dict(Nx=32, Ny=32), dict(Nx=20, Ny=12, x0=-1.0, x1=2.0, gamma=5.0 / 3.0, seed=7)):
        p = ParamsNS(**kw)
        cp = p.to_c()
        got = ic_collapse(p)
        want = [np.zeros(p.Nx * p.Ny) for _ in range(4)]
        O.oracle().or_ns2d_ic(C.byref(cp), O.pp(want))
        for x, y in zip(got.arrays(), want):
            assert np.array_equal(x, y)
    # the IC's statistics: unit background with a Gaussian bump, P = 0.05
    p = ParamsNS(Nx=64, Ny=64)
    s = ic_collapse(p)
    P = (p.gamma - 1.0) * (s.E - 0.5 * (s.mx**2 + s.my**2) / s.rho)
    assert np.allclose(P, 0.05, rtol=1e-12)
    r = s.rho.reshape(64, 64)
    assert 1.9 < r[31:33, 31:33].mean() < 2.1 and 0.95 < r[0, :].mean() < 1.05


def test_fft_potential_of_rhs_matches_reference_solver():
    """The oracle's gravity (spectral phi and g, NS:285-360) equals the
    reference's solve_poisson_periodic_fft + compute_gravity_accel."""
    R = O.ref("fft")
    if R is None:
        pytest.skip("compiled reference (oracle/_ref) not available")
    p, s = make_case_ns("kicked_viscous")
    cp = p.to_c()
    n = p.Nx * p.Ny
    phi, gx, gy = np.zeros(n), np.zeros(n), np.zeros(n)
    O.oracle().or_ns2d_gravity(C.byref(cp), O.pp(s.arrays()), O.dp(phi), O.dp(gx), O.dp(gy))
    rho = np.maximum(s.rho, p.floor_rho)
    phr, gxr, gyr = np.zeros(n), np.zeros(n), np.zeros(n)
    R.ref_fft_poisson(p.Nx, p.Ny, p.x0, p.x1, p.y0, p.y1, p.G, O.dp(rho), O.dp(phr))
    R.ref_fft_gravity_accel(p.Nx, p.Ny, p.x0, p.x1, p.y0, p.y1, O.dp(phr), O.dp(gxr), O.dp(gyr))
    assert np.array_equal(phi, phr) and np.array_equal(gx, gxr) and np.array_equal(gy, gyr)
