"""Seeded 2D Navier-Stokes cases shared by the oracle pin tests and the GPU
parity tests: the reference's collapse IC (NS:627-689) and kicked variants
that reach every HLLC branch, strong viscous stresses and the floors."""
from __future__ import annotations

import zlib

import numpy as np

from core_collapse_b200.ns2d import ParamsNS, StateNS, ic_collapse

CASES_NS = {
    # the reference main()'s parameters and IC on a small grid
    "collapse_ic": dict(p=dict(Nx=32, Ny=32), kick=0.0),
    # supersonic kicks both ways (every HLLC branch), strong viscosity, non-square box
    "kicked_viscous": dict(p=dict(Nx=32, Ny=16, x0=-1.0, x1=1.0, y0=0.0, y1=0.5, gamma=5.0 / 3.0, mu=2e-3,
                                  G=4.0), kick=2.0),
    # inviscid, no gravity, grid sizes that are not powers of two
    "inviscid_nograv_odd": dict(p=dict(Nx=20, Ny=12, viscosity_on=False, gravity_on=False), kick=1.5),
    # viscous without gravity, mu > 0
    "viscous_nograv": dict(p=dict(Nx=24, Ny=16, gravity_on=False, mu=5e-3), kick=0.8),
    # density and pressure below their floors in a patch
    "floors": dict(p=dict(Nx=32, Ny=16, floor_rho=1e-3, floor_P=1e-3, mu=1e-3), kick=0.5, floor_patch=True),
}


def make_case_ns(name: str, precision: str = "fp64") -> tuple[ParamsNS, StateNS]:
    c = CASES_NS[name]
    p = ParamsNS(**c["p"], precision=precision)
    s = ic_collapse(p)
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if c["kick"] > 0.0:
        n = p.Nx * p.Ny
        u = c["kick"] * rng.uniform(-1.0, 1.0, n)
        v = c["kick"] * rng.uniform(-1.0, 1.0, n)
        ke_old = 0.5 * (s.mx**2 + s.my**2) / s.rho
        s.mx = s.rho * u
        s.my = s.rho * v
        s.E = s.E - ke_old + 0.5 * s.rho * (u * u + v * v)
    if c.get("floor_patch"):
        r = s.rho.reshape(p.Ny, p.Nx)
        E = s.E.reshape(p.Ny, p.Nx)
        r[2:5, 3:9] = 1e-5           # below floor_rho
        E[6:9, 10:14] = 1e-6          # pressure below floor_P
        s.rho, s.E = r.ravel().copy(), E.ravel().copy()
    return p, s
