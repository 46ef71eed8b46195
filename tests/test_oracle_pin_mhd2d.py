"""Pin the CPU restatement (oracle/) to the reference itself.

The reference solver sources are compiled in place into oracle/_ref/ (see
oracle/Makefile) and run here on the same seeded inputs; the restatement must
reproduce them bit for bit (both are FP64 without FMA, same operation order).
Skipped where the compiled reference is absent (it is built from the
reference tree, which only this container has)."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_mhd2d import CASES, make_case

pytestmark = pytest.mark.skipif(O.ref("mhd2d") is None, reason="compiled reference (oracle/_ref) not available")


def _setup(name):
    p, U, B = make_case(name)
    cp = p.to_c()
    S = O.state_list(U, B)
    n = p.Nx * p.Ny
    gx, gy = np.zeros(n), np.zeros(n)
    if p.gravity_on:
        O.ref("mhd2d").ref_mhd2d_poisson(C.byref(cp), O.dp(S[0]), O.dp(gx), O.dp(gy))
    dt = O.ref("mhd2d").ref_mhd2d_compute_dt(C.byref(cp), O.pp(S))
    return p, cp, S, gx, gy, dt


@pytest.mark.parametrize("name", sorted(CASES))
def test_compute_dt_bitwise(name):
    p, cp, S, gx, gy, dt = _setup(name)
    assert O.oracle().or_mhd2d_compute_dt(C.byref(cp), O.pp(S)) == dt


@pytest.mark.parametrize("name", sorted(CASES))
def test_advance_stage_bitwise(name):
    p, cp, S, gx, gy, dt = _setup(name)
    a = O.m2_stage_ref(cp, S, gx, gy, dt)
    b = O.m2_stage_oracle(cp, S, gx, gy, dt)
    for k, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"field {k} differs, max |d| = {np.max(np.abs(x - y))}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_rk2_step_bitwise(name):
    p, cp, S, gx, gy, dt = _setup(name)
    a = O.m2_rk2_ref(cp, S, gx, gy, dt)
    b = O.m2_rk2_oracle(cp, S, gx, gy, dt, mode=0)
    for k, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"field {k} differs, max |d| = {np.max(np.abs(x - y))}"


@pytest.mark.parametrize("name", ["periodic_grav_eta", "outflow_grav_eta", "mixed_ot_ideal"])
def test_main_loop_bitwise(name):
    p, cp, S, gx, gy, dt = _setup(name)
    cp.t_end = 10.0
    a = O.copy_state(S)
    t = C.c_double(0.0)
    O.ref("mhd2d").ref_mhd2d_main_loop(C.byref(cp), O.pp(a), 3, C.byref(t))
    b, tb = O.m2_main_loop_oracle(cp, S, 3, mode=0)
    assert t.value == tb
    for k, (x, y) in enumerate(zip(a, b)):
        assert np.array_equal(x, y), f"field {k} differs"


@pytest.mark.parametrize("periodic", [True, False])
def test_sor_fixed_sweeps_bitwise(periodic):
    name = "periodic_grav_eta" if periodic else "outflow_grav_eta"
    p, cp, S, gx, gy, dt = _setup(name)
    ox, oy, it, res = O.m2_gravity_oracle(cp, S[0], mode=0)
    assert it == p.sor_iters
    assert np.array_equal(ox, gx) and np.array_equal(oy, gy)


def test_sor_tolerance_matches_euler2d_reference():
    """Restated tolerance SOR == euler2d_gravity_hllc.cpp:288-386 (omega 1.7,
    tol 1e-10, floored density, periodic), bit for bit."""
    R = O.ref("euler2d")
    if R is None:
        pytest.skip("euler2d reference not built")
    from core_collapse_b200 import _lib as L
    cp = L.CcEuler2dParams(gamma=1.2, cfl=0.45, x0=0.0, x1=1.0, y0=0.0, y1=1.0, Nx=16, Ny=12, t_end=5.0,
                           dt_store=1e-3, floor_rho=1e-12, floor_P=1e-12, periodic_x=1, periodic_y=1, gravity_on=1,
                           sor_max_iter=50000, G=1.0, softening=1e-4, sor_tol=1e-10, sor_omega=1.7)
    n = 16 * 12
    f = [np.zeros(n) for _ in range(4)]
    R.ref_euler2d_init_random_blob(C.byref(cp), O.pp(f))
    gx, gy = np.zeros(n), np.zeros(n)
    R.ref_euler2d_poisson(C.byref(cp), O.pp(f), O.dp(gx), O.dp(gy))
    ox, oy = np.zeros(n), np.zeros(n)
    it, res = C.c_int(), C.c_double()
    O.oracle().or_poisson_generic(16, 12, 1, 1, 1.0 / 16, 1.0 / 12, 1.0, 1.7, 50000, 1e-10, 1, 1e-12, 0,
                                  O.dp(f[0]), O.dp(ox), O.dp(oy), C.byref(it), C.byref(res))
    assert res.value < 1e-10 and 0 < it.value < 50000
    assert np.array_equal(ox, gx) and np.array_equal(oy, gy)


@pytest.mark.parametrize("periodic", [True, False])
def test_red_black_converges_to_lexicographic(periodic):
    """The GPU ordering (red-black) and the reference ordering converge to the
    same discrete solution: at tol 1e-11 the two g fields agree to ~1e-9."""
    name = "periodic_grav_eta" if periodic else "outflow_grav_eta"
    p, U, B = make_case(name)
    p.sor_tol = 1e-11
    p.sor_iters = 200000
    cp = p.to_c()
    lx, ly, itl, rl = O.m2_gravity_oracle(cp, U.rho, mode=0)
    bx, by, itb, rb = O.m2_gravity_oracle(cp, U.rho, mode=1)
    assert rl < 1e-11 and rb < 1e-11
    assert O.rel_linf(bx, lx) < 1e-8 and O.rel_linf(by, ly) < 1e-8


def test_fft1d_bitwise():
    R = O.ref("fft")
    rng = np.random.default_rng(11)
    for n in (2, 8, 64, 256):
        for inv in (0, 1):
            z = rng.normal(size=2 * n)
            a, b = z.copy(), z.copy()
            R.ref_fft1d(n, O.dp(a), inv)
            O.oracle().or_fft1d(n, O.dp(b), inv)
            assert np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(16, 16), (32, 8), (8, 64)])
def test_fft_poisson_bitwise(shape):
    """Restated spectral solve == navier_stokes_2d_hllc_poisson.cpp:285-328."""
    R = O.ref("fft")
    nx, ny = shape
    rng = np.random.default_rng(nx * 1000 + ny)
    rho = 1.0 + rng.random(nx * ny)
    phi_ref = np.zeros(nx * ny)
    R.ref_fft_poisson(nx, ny, -1.0, 1.0, -1.0, 1.0, 1.0, O.dp(rho), O.dp(phi_ref))
    from core_collapse_b200.mhd2d import Params
    p = Params(Nx=nx, Ny=ny, x0=-1, x1=1, y0=-1, y1=1, G=1.0, poisson="fft")
    cp = p.to_c()
    phi = np.zeros(nx * ny)
    O.oracle().or_mhd2d_phi(C.byref(cp), O.dp(rho), O.dp(phi), 2, None, None)
    assert np.array_equal(phi, phi_ref)
