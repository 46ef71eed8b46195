"""Seeded small 2D MHD cases shared by the CPU pin tests, the golden-fixture
script and the GPU parity tests.  Each case perturbs a library IC so that
every branch of the step is reached: HLLD star and double-star regions, the
|Bn|<1e-12 HLL fallback, supersonic upwind faces, limiter clipping, pressure
floors, both boundary kinds and both wrap rules of the face arrays."""
from __future__ import annotations

import numpy as np

from core_collapse_b200.mhd2d import Params, ic_collapse, ic_orszag_tang, ic_reference

CASES = {
    # name: (Params kwargs, IC kind, IC kwargs, perturbation seed)
    "periodic_grav_eta": (dict(Nx=12, Ny=10, x0=-1, x1=1, y0=-1, y1=1, periodic_x=True, periodic_y=True, eta=1e-3,
                               gravity_on=True, G=1.0, sor_iters=40, sor_omega=1.9, cfl=0.4),
                          "collapse", dict(core_amp=9.0, core_width=0.3, noise=0.01, seed=0, Bx0=0.05), 1),
    "outflow_grav_eta": (dict(Nx=9, Ny=7, x0=-1, x1=1, y0=-1, y1=1, periodic_x=False, periodic_y=False, eta=1e-3,
                              gravity_on=True, G=1.0, sor_iters=40, sor_omega=1.9, cfl=0.4),
                         "collapse", dict(core_amp=9.0, core_width=0.4, noise=0.01, seed=0, Bx0=0.05), 2),
    "mixed_ot_ideal": (dict(Nx=8, Ny=12, x0=-1, x1=1, y0=-1, y1=1, periodic_x=True, periodic_y=False, eta=0.0,
                            gravity_on=False, cfl=0.4),
                       "ot", dict(core_amp=4.0, core_width=0.3), 3),
    "reference_ic": (dict(Nx=16, Ny=16, periodic_x=True, periodic_y=True, eta=5e-4, gravity_on=True, G=8.0,
                          sor_iters=30, sor_omega=1.8, cfl=0.45),
                     "reference", dict(r_core=0.25, r_edge=0.05), 4),
    "hll_fallback_outflow": (dict(Nx=10, Ny=10, x0=-1, x1=1, y0=-1, y1=1, periodic_x=False, periodic_y=True,
                                  eta=2e-3, gravity_on=True, G=1.0, sor_iters=20, sor_omega=1.9, cfl=0.4),
                             "collapse", dict(core_amp=5.0, core_width=0.4, noise=0.05, seed=7, Bx0=0.0), 5),
}


def make_case(name: str, precision: str = "fp64", poisson: str = "sor"):
    kw, kind, ickw, seed = CASES[name]
    p = Params(**kw, precision=precision, poisson=poisson)
    if kind == "collapse":
        U, B = ic_collapse(p, **ickw)
    elif kind == "ot":
        U, B = ic_orszag_tang(p, **ickw)
    else:
        U, B = ic_reference(p, **ickw)
    rng = np.random.default_rng(seed)
    n = p.Nx * p.Ny
    # velocity kicks (some supersonic), a transverse field and Bz, a few cold cells
    U.mx += U.rho * rng.normal(0.0, 0.6, n)
    U.my += U.rho * rng.normal(0.0, 0.6, n)
    U.mz += U.rho * rng.normal(0.0, 0.2, n)
    U.Bz += rng.normal(0.0, 0.05, n)
    kin = 0.5 * (U.mx ** 2 + U.my ** 2 + U.mz ** 2) / U.rho
    U.E += kin + 0.5 * U.Bz ** 2
    cold = rng.choice(n, size=max(1, n // 15), replace=False)
    U.E[cold] = 0.5 * (U.mx[cold] ** 2 + U.my[cold] ** 2 + U.mz[cold] ** 2) / U.rho[cold]
    return p, U, B
