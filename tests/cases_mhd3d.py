"""Seeded small 3D MHD cases for the pin and GPU parity tests.  Faces come
from a random edge vector potential through the discrete curl, so div B is
zero to roundoff; densities are spread so that the hybrid-EOS cases cross
rho_nuc (80) and rho_bounce (120)."""
from __future__ import annotations

import numpy as np

from core_collapse_b200.mhd3d import Params3, State3

CASES3 = {
    # name: (Params3 constructor kwargs, ideal-gas mapping?, dense cells?, seed)
    "periodic_ideal": (dict(Nx=6, Ny=5, Nz=4, eta=5e-4, cfl=0.4), True, False, 1),
    "outflow_ideal": (dict(Nx=5, Ny=6, Nz=5, periodic_x=False, periodic_y=False, periodic_z=False, eta=1e-3),
                      True, False, 2),
    "mixed_hybrid": (dict(Nx=6, Ny=4, Nz=5, periodic_x=True, periodic_y=False, periodic_z=True, eta=5e-4),
                     False, True, 3),
    "periodic_hybrid_ideal_mhd": (dict(Nx=4, Ny=6, Nz=6, eta=0.0), False, True, 4),
}


def make_case3(name: str, precision: str = "fp64", periodic_potential: bool = False):
    """periodic_potential: make the edge potential periodic along periodic axes,
    so that faces 0 and N carry the same B (the reference evolves them as
    separate values; with a non-periodic potential they differ and fluxes
    through the seam do not cancel)."""
    kw, ideal, dense, seed = CASES3[name]
    p = Params3.ideal_gas(**kw, precision=precision) if ideal else Params3(**kw, precision=precision)
    rng = np.random.default_rng(seed)
    nx, ny, nz = p.Nx, p.Ny, p.Nz
    n = nx * ny * nz
    # edge vector potential -> face B = curl A (+ uniform field)
    Ax = rng.normal(0, 0.05, (nz + 1, ny + 1, nx))
    Ay = rng.normal(0, 0.05, (nz + 1, ny, nx + 1))
    Az = rng.normal(0, 0.05, (nz, ny + 1, nx + 1))
    if periodic_potential:
        for A in (Ax, Ay, Az):
            if p.periodic_x and A.shape[2] == nx + 1:
                A[:, :, nx] = A[:, :, 0]
            if p.periodic_y and A.shape[1] == ny + 1:
                A[:, ny, :] = A[:, 0, :]
            if p.periodic_z and A.shape[0] == nz + 1:
                A[nz, :, :] = A[0, :, :]
    dx, dy, dz = p.dx, p.dy, p.dz
    bx = (Az[:, 1:, :] - Az[:, :-1, :]) / dy - (Ay[1:, :, :] - Ay[:-1, :, :]) / dz + 0.15
    by = (Ax[1:, :, :] - Ax[:-1, :, :]) / dz - (Az[:, :, 1:] - Az[:, :, :-1]) / dx
    bz = (Ay[:, :, 1:] - Ay[:, :, :-1]) / dx - (Ax[:, 1:, :] - Ax[:, :-1, :]) / dy + 0.05
    rho = 1.0 + 2.0 * rng.random(n)
    if dense:
        idx = rng.choice(n, size=max(3, n // 6), replace=False)
        rho[idx[: len(idx) // 2]] = 90.0 + 20.0 * rng.random(len(idx) // 2)      # above rho_nuc
        rho[idx[len(idx) // 2:]] = 125.0 + 30.0 * rng.random(len(idx) - len(idx) // 2)  # above rho_bounce
    u, v, w = (rng.normal(0, 0.5, n) for _ in range(3))
    P = 0.5 + rng.random(n)
    bxc = 0.5 * (bx[:, :, :-1] + bx[:, :, 1:]).ravel()
    byc = 0.5 * (by[:, :-1, :] + by[:, 1:, :]).ravel()
    bzc = 0.5 * (bz[:-1, :, :] + bz[1:, :, :]).ravel()
    E = 0.5 * rho * (u * u + v * v + w * w) + 0.5 * (bxc ** 2 + byc ** 2 + bzc ** 2) + P / (p.gamma_th - 1.0)
    cold = rng.choice(n, size=max(1, n // 20), replace=False)
    E[cold] = 0.5 * rho[cold] * (u[cold] ** 2 + v[cold] ** 2 + w[cold] ** 2)
    s = State3(rho, rho * u, rho * v, rho * w, E, bx.ravel().copy(), by.ravel().copy(), bz.ravel().copy())
    return p, s
