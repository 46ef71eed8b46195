"""Pin the 2D Euler/HLLC restatement (oracle/euler2d_oracle.hpp) to the
reference euler2d_gravity_hllc.cpp compiled in place: bit-identical rhs (with
the reference's own tolerance SOR inside), compute_dt, rk2_step and main-loop
steps, on the reference's own random-blob IC and on seeded kicked cases."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_euler2d import CASES_EH, make_case_eh

pytestmark = pytest.mark.skipif(O.ref("euler2d") is None, reason="compiled reference (oracle/_ref) not available")


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_rhs_dt_and_step_bitwise(name):
    p, s = make_case_eh(name)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    R = O.ref("euler2d")
    assert O.oracle().or_euler2d_compute_dt(C.byref(cp), O.pp(S)) == R.ref_euler2d_compute_dt(C.byref(cp), O.pp(S))
    a = [np.zeros_like(x) for x in S]
    b = [np.zeros_like(x) for x in S]
    R.ref_euler2d_rhs(C.byref(cp), O.pp(S), O.pp(a))
    O.oracle().or_euler2d_rhs(C.byref(cp), O.pp(S), O.pp(b), 0)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    dt = R.ref_euler2d_compute_dt(C.byref(cp), O.pp(S))
    a = O.copy_state(S)
    b = O.copy_state(S)
    R.ref_euler2d_rk2_step(C.byref(cp), O.pp(a), dt)
    O.oracle().or_euler2d_rk2_step(C.byref(cp), O.pp(b), dt, 0)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_random_blob_main_loop_bitwise():
    """The reference's own IC (EH:574-642) and main-loop body, 3 steps."""
    from core_collapse_b200.euler2d import ParamsEH
    p = ParamsEH(Nx=20, Ny=16)
    cp = p.to_c()
    n = p.Nx * p.Ny
    R = O.ref("euler2d")
    S = [np.zeros(n) for _ in range(4)]
    R.ref_euler2d_init_random_blob(C.byref(cp), O.pp(S))
    a = O.copy_state(S)
    t = C.c_double(0.0)
    assert R.ref_euler2d_main_loop(C.byref(cp), O.pp(a), 3, C.byref(t)) == 0
    b, tb, rc = O.eh_main_loop_oracle(cp, S, 3, mode=0)
    assert rc == 0 and tb == t.value
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_library_random_blob_ic_equals_reference():
    """cc_ic_euler2d_random_blob reproduces init_random_blob (EH:574-642) bit for bit."""
    from core_collapse_b200.euler2d import ParamsEH, ic_random_blob
    for kw in (dict(Nx=20, Ny=16), dict(Nx=7, Ny=9, x0=-1.0, x1=2.0, gamma=1.4)):
        p = ParamsEH(**kw)
        cp = p.to_c()
        n = p.Nx * p.Ny
        S = [np.zeros(n) for _ in range(4)]
        O.ref("euler2d").ref_euler2d_init_random_blob(C.byref(cp), O.pp(S))
        U = ic_random_blob(p)
        for a, b in zip(U.arrays(), S):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_enclosed_mass_gravity_bitwise(name):
    """The oracle's enclosed-mass gravity == compute_enclosed_mass_gravity of the
    compiled reference (EH:226-286), bit for bit (same sort, same summation order);
    square grids give many equal radii, so the tie grouping is exercised."""
    from core_collapse_b200 import _lib as L
    p, s = make_case_eh(name)
    p.poisson = "enclosed"
    cp = p.to_c()
    cp.gravity_on = 1
    cp.poisson_kind = L.CC_GRAVITY_ENCLOSED
    S = [a.copy() for a in s.arrays()]
    n = p.Nx * p.Ny
    gx, gy, hx, hy = (np.zeros(n) for _ in range(4))
    O.ref("euler2d").ref_euler2d_enclosed_gravity(C.byref(cp), O.pp(S), O.dp(gx), O.dp(gy))
    O.oracle().or_euler2d_gravity(C.byref(cp), O.dp(S[0]), O.dp(hx), O.dp(hy), 0, None, None)
    assert np.array_equal(gx, hx) and np.array_equal(gy, hy)
    assert np.max(np.abs(gx)) > 0


@pytest.mark.parametrize("name", sorted(CASES_EH))
@pytest.mark.parametrize("knobs", [dict(Nr_bins=512), dict(Nr_bins=3, xc=0.3, yc=0.8), dict(Nr_bins=64, xc=-0.2)])
def test_shell_gravity_bitwise(name, knobs):
    """The oracle's shell-binned enclosed-mass gravity == the compiled
    gravity_accel_from_enclosed_mass (gravity_enclosed.h:18-96), bit for bit:
    shells at least 8, centres inside and outside the box."""
    from core_collapse_b200 import _lib as L
    if O.ref("ge") is None:
        pytest.skip("compiled reference (oracle/_ref) not available")
    p, s = make_case_eh(name)
    for k, v in knobs.items():
        setattr(p, k, v)
    p.gravity_on, p.poisson = True, "shells"
    cp = p.to_c()
    n = p.Nx * p.Ny
    gx, gy, hx, hy = (np.zeros(n) for _ in range(4))
    O.ref("ge").ref_ge_gravity(p.Nx, p.Ny, p.x0, p.x1, p.y0, p.y1, p.G, p.softening, p.Nr_bins, p.xc, p.yc,
                               p.floor_rho, O.dp(s.rho.copy()), O.dp(gx), O.dp(gy))
    O.oracle().or_euler2d_gravity(C.byref(cp), O.dp(s.rho.copy()), O.dp(hx), O.dp(hy), 0, None, None)
    assert cp.poisson_kind == L.CC_GRAVITY_SHELLS
    assert np.array_equal(gx, hx) and np.array_equal(gy, hy)
    assert np.max(np.abs(gx)) > 0


def test_shell_gravity_centre_cell_without_softening():
    """A cell centre exactly at the gravity centre with softening 0: the
    reference's denom <= 0 branch gives g = 0 there."""
    from core_collapse_b200.euler2d import ParamsEH
    if O.ref("ge") is None:
        pytest.skip("compiled reference (oracle/_ref) not available")
    p = ParamsEH(Nx=9, Ny=9, softening=0.0, poisson="shells", gravity_on=True)
    cp = p.to_c()
    rho = np.linspace(0.5, 2.0, 81)
    gx, gy, hx, hy = (np.zeros(81) for _ in range(4))
    O.ref("ge").ref_ge_gravity(9, 9, 0.0, 1.0, 0.0, 1.0, p.G, 0.0, p.Nr_bins, 0.5, 0.5, p.floor_rho, O.dp(rho),
                               O.dp(gx), O.dp(gy))
    O.oracle().or_euler2d_gravity(C.byref(cp), O.dp(rho), O.dp(hx), O.dp(hy), 0, None, None)
    assert np.array_equal(gx, hx) and np.array_equal(gy, hy) and gx[40] == 0.0 and gy[40] == 0.0
