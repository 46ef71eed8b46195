"""The lexicographic SOR parity mode (CC_POISSON_SOR_LEX, sor_lex_kernel in
poisson_kernels.cuh) against the oracle's restatement of the reference's own
solve (mode 0: the row-major sweep and sequential means of M2:178-237, pinned
bit for bit to the compiled reference by the oracle pin tests).  FP64: the
gravity field and the main-loop steps are the same doubles, on every seeded
gravity case (periodic, outflow and mixed axes, the reference IC, the HLL
fallback case) and on odd periodic extents, which the red-black ordering
cannot take.  FP32 (density read as FP32, the solve in FP64) is checked
against the same oracle with the FP32 bound of the other gravity tests.
Euler/HLLC (EH:288-386: floored density, the reference's residual tolerance
1e-10 taken inside the sweep, an always-periodic stencil): the same gravity,
sweep count and residual, and the same RK2 step, bit for bit."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_euler2d import CASES_EH, make_case_eh
from cases_mhd2d import CASES, make_case
from core_collapse_b200.euler2d import Euler2dSolver
from core_collapse_b200.mhd2d import Mhd2dSolver, Params, ic_collapse

pytestmark = pytest.mark.gpu

GRAV_CASES = [n for n in sorted(CASES) if CASES[n][0].get("gravity_on")]


def _gravity(p, U, B):
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        g = s.compute_gravity()
        d = s.diagnostics()
    return g, d


@pytest.mark.parametrize("name", GRAV_CASES)
def test_gravity_lex_bit_identical(name):
    p, U, B = make_case(name, poisson="sor_lex")
    gx, gy, it, _ = O.m2_gravity_oracle(p.to_c(), U.rho, mode=0)
    g, d = _gravity(p, U, B)
    assert d["poisson_iters"] == it == p.sor_iters
    assert np.array_equal(g.gx, gx) and np.array_equal(g.gy, gy)


@pytest.mark.parametrize("shape,periodic", [((37, 23), (True, True)), ((2, 9), (True, False)), ((40, 3), (False, True))])
def test_gravity_lex_odd_and_thin_grids(shape, periodic):
    nx, ny = shape
    p = Params(Nx=nx, Ny=ny, x0=-1, x1=1, y0=-1, y1=1, periodic_x=periodic[0], periodic_y=periodic[1],
               gravity_on=True, G=1.0, sor_iters=25, sor_omega=1.8, poisson="sor_lex")
    U, B = ic_collapse(p, core_amp=6.0, core_width=0.3, noise=0.02, seed=3, Bx0=0.05)
    gx, gy, _, _ = O.m2_gravity_oracle(p.to_c(), U.rho, mode=0)
    g, _ = _gravity(p, U, B)
    assert np.array_equal(g.gx, gx) and np.array_equal(g.gy, gy)


@pytest.mark.parametrize("name", GRAV_CASES)
def test_main_loop_lex_bit_identical(name):
    p, U, B = make_case(name, poisson="sor_lex")
    p.t_end = 10.0
    want, t_want = O.m2_main_loop_oracle(p.to_c(), O.state_list(U, B), 4, mode=0)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        t = s.advance(4, 0.0)
        got = O.state_list(*s.download())
    assert t == t_want
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"field {k}: max |d| {np.max(np.abs(a - b)):.3e}"


def test_gravity_lex_tolerance_stops_like_oracle():
    p, U, B = make_case("periodic_grav_eta", poisson="sor_lex")
    p.sor_tol, p.sor_iters = 1e-9, 100000
    gx, gy, it, _ = O.m2_gravity_oracle(p.to_c(), U.rho, mode=0)
    g, d = _gravity(p, U, B)
    assert d["poisson_iters"] == it and d["poisson_residual"] < 1e-9
    assert np.array_equal(g.gx, gx) and np.array_equal(g.gy, gy)


def test_gravity_lex_fp32():
    p, U, B = make_case("outflow_grav_eta", precision="fp32", poisson="sor_lex")
    gx, gy, _, _ = O.m2_gravity_oracle(p.to_c(), U.rho, mode=0)
    g, _ = _gravity(p, U, B)
    assert O.rel_linf(g.gx, gx) <= 2e-5 and O.rel_linf(g.gy, gy) <= 2e-5


# ---- Euler/HLLC ----

EH_GRAV = [n for n in sorted(CASES_EH) if CASES_EH[n][0].get("gravity_on")]


@pytest.mark.parametrize("name", EH_GRAV)
def test_euler_gravity_lex_bit_identical(name):
    p, s = make_case_eh(name, poisson="sor_lex")   # the reference's tolerance 1e-10
    cp = p.to_c()
    n = p.Nx * p.Ny
    gx, gy = np.zeros(n), np.zeros(n)
    it, res = C.c_int(), C.c_double()
    O.oracle().or_euler2d_gravity(C.byref(cp), O.dp(s.rho), O.dp(gx), O.dp(gy), 0, C.byref(it), C.byref(res))
    with Euler2dSolver(p) as g:
        g.upload(s)
        x, y = g.compute_gravity()
        d = g.diagnostics()
    assert d["poisson_iters"] == it.value and d["poisson_residual"] == res.value
    assert np.array_equal(x, gx) and np.array_equal(y, gy)


@pytest.mark.parametrize("name", EH_GRAV)
def test_euler_rk2_step_lex_bit_identical(name):
    p, s = make_case_eh(name, poisson="sor_lex")
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    dt = O.oracle().or_euler2d_compute_dt(C.byref(cp), O.pp(S))
    want = O.copy_state(S)
    O.oracle().or_euler2d_rk2_step(C.byref(cp), O.pp(want), dt, 0)
    with Euler2dSolver(p) as g:
        g.upload(s)
        g.rk2_step(dt)
        got = g.download().arrays()
    for a, b in zip(got, want):
        assert np.array_equal(a, b)
