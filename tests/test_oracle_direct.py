"""CPU checks of the oracle's direct Poisson solve (mode 3), the restatement
the batched ensemble's GPU solve is compared with bit for bit.

It must be the problem the reference's SOR solves (M2:207-223): its residual
max|lap(phi) - rhs| is at roundoff, and red-black SOR iterated to 1e-13
converges to it, on clamp, periodic and mixed boundaries."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_mhd2d import make_case
from core_collapse_b200.mhd2d import Params


@pytest.mark.parametrize("name", ["periodic_grav_eta", "outflow_grav_eta", "hll_fallback_outflow"])
def test_direct_equals_converged_sor(name):
    p, U, B = make_case(name)
    p.sor_tol = 1e-13
    p.sor_iters = 400000
    cp = p.to_c()
    sx, sy, _, _ = O.m2_gravity_oracle(cp, U.rho, mode=1)
    dx, dy, _, res = O.m2_gravity_oracle(cp, U.rho, mode=3)
    assert res < 1e-11
    assert O.rel_linf(dx, sx) < 1e-13 and O.rel_linf(dy, sy) < 1e-13


@pytest.mark.parametrize("px,py", [(False, False), (True, True), (True, False), (False, True)])
def test_direct_solve_is_the_dense_discrete_solution(px, py):
    """Against numpy's least-squares solve of the assembled 5-point system with
    the zero-mean constraint (a dense restatement of the same problem)."""
    nx, ny = 10, 7
    p = Params(Nx=nx, Ny=ny, x0=-1, x1=1, y0=-1, y1=2, periodic_x=px, periodic_y=py, G=1.3, poisson="direct")
    rng = np.random.default_rng(5)
    rho = 1.0 + rng.random(nx * ny)
    phi = np.zeros(nx * ny)
    O.oracle().or_mhd2d_phi(C.byref(p.to_c()), O.dp(rho), O.dp(phi), 3, None, None)
    ax = lambda i: i % nx if px else min(max(i, 0), nx - 1)
    ay = lambda j: j % ny if py else min(max(j, 0), ny - 1)
    A = np.zeros((nx * ny + 1, nx * ny))
    for j in range(ny):
        for i in range(nx):
            r = j * nx + i
            for (ii, jj, w) in ((i + 1, j, 1 / p.dx ** 2), (i - 1, j, 1 / p.dx ** 2), (i, j + 1, 1 / p.dy ** 2),
                                (i, j - 1, 1 / p.dy ** 2)):
                A[r, ay(jj) * nx + ax(ii)] += w
                A[r, r] -= w
    A[-1, :] = 1.0
    rhs = np.append(4 * np.pi * p.G * (rho - rho.mean()), 0.0)
    want = np.linalg.lstsq(A, rhs, rcond=None)[0]
    assert np.max(np.abs(phi - want)) <= 1e-11 * np.max(np.abs(want))
