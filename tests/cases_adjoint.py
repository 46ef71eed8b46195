"""Seeded 2D MHD states for the adjoint tests (GPU adjoint, oracle tangent).

Collapse core with velocity kicks, Bz noise and an in-plane B made of a
uniform (0.1, 0.07) plus the curl of a random corner potential (div B = 0 to
roundoff), so that no face sits on the HLL branch (Bn = 0) and no MC slope on
its zero kink: finite differences then measure derivatives."""
import numpy as np

from core_collapse_b200.mhd2d import Params, ic_collapse


def make_case_adj(periodic: bool, grav: bool, nx=24, ny=20, eta=2e-3, seed=3):
    p = Params(Nx=nx, Ny=ny, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=periodic, periodic_y=not periodic,
               gamma=5.0 / 3.0, G=1.0, eta=eta, cfl=0.4, gravity_on=grav, poisson="direct", t_end=1e30)
    U, B = ic_collapse(p, core_amp=6.0, core_width=0.3, noise=0.02, seed=seed, Bx0=0.1)
    rng = np.random.default_rng(seed)
    n = nx * ny
    U.mx += U.rho * rng.normal(0.0, 0.3, n)
    U.my += U.rho * rng.normal(0.0, 0.3, n)
    U.mz += U.rho * rng.normal(0.0, 0.1, n)
    U.Bz += rng.normal(0.0, 0.05, n)
    # In-plane B = uniform (0.1, 0.07) + curl of a random corner potential
    # Az (div B = 0 to roundoff).  A finite-difference step must not sit on a
    # branch point of the discrete map: Bn = 0 selects HLL (|Bn| < 1e-12,
    # M2:449) and a uniform field gives zero MC slopes, the limiter's kink.
    Az = rng.normal(0.0, 0.004, (ny + 1, nx + 1))
    B.Bx_f[:] = (0.1 + (Az[1:, :] - Az[:-1, :]) / p.dy).ravel()
    B.By_f[:] = (0.07 - (Az[:, 1:] - Az[:, :-1]) / p.dx).ravel()
    Bx = 0.5 * (B.Bx_f.reshape(ny, nx + 1)[:, 1:] + B.Bx_f.reshape(ny, nx + 1)[:, :-1]).ravel()
    By = 0.5 * (B.By_f.reshape(ny + 1, nx)[1:, :] + B.By_f.reshape(ny + 1, nx)[:-1, :]).ravel()
    U.E += 0.5 * (U.mx ** 2 + U.my ** 2 + U.mz ** 2) / U.rho + 0.5 * (U.Bz ** 2 + Bx ** 2 + By ** 2) - 0.5 * 0.01
    return p, U, B
