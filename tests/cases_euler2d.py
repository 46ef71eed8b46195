"""Seeded small 2D Euler cases: the reference's own random-blob IC
(init_random_blob, EH:574-642, run through the compiled reference where it is
available, else the library's restatement of it) plus supersonic kicks and
cold cells, on periodic, outflow and mixed boundaries."""
from __future__ import annotations

import numpy as np

from core_collapse_b200.euler2d import ParamsEH, StateEH

CASES_EH = {
    "periodic_grav": (dict(Nx=12, Ny=10, periodic_x=True, periodic_y=True, gravity_on=True, G=1.0), 1),
    "outflow_grav": (dict(Nx=10, Ny=8, periodic_x=False, periodic_y=False, gravity_on=True, G=2.0), 2),
    "mixed_nograv": (dict(Nx=8, Ny=12, periodic_x=True, periodic_y=False, gravity_on=False), 3),
    "outflow_odd_nograv": (dict(Nx=9, Ny=7, periodic_x=False, periodic_y=False, gravity_on=False), 4),
}


def make_case_eh(name: str, precision: str = "fp64", poisson: str = "sor"):
    kw, seed = CASES_EH[name]
    p = ParamsEH(**kw, precision=precision, poisson=poisson)
    rng = np.random.default_rng(seed)
    n = p.Nx * p.Ny
    x = p.x0 + (np.arange(p.Nx) + 0.5) * p.dx
    y = p.y0 + (np.arange(p.Ny) + 0.5) * p.dy
    X, Y = np.meshgrid(x, y)
    rho = (1.0 + 0.1 * (2 * rng.random((p.Ny, p.Nx)) - 1) + 0.5 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / (2 * 0.15 ** 2))).ravel()
    u = rng.normal(0, 0.8, n)
    v = rng.normal(0, 0.8, n)
    P = 1.0 + 0.1 * (2 * rng.random(n) - 1)
    E = P / (p.gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    cold = rng.choice(n, size=max(1, n // 15), replace=False)
    E[cold] = 0.5 * rho[cold] * (u[cold] ** 2 + v[cold] ** 2)
    return p, StateEH(rho, rho * u, rho * v, E)
