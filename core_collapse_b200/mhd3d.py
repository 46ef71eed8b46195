"""3D resistive MHD on the GPU, behind the reference's own interface
(mhd3d_resistive_hlld_ct.cpp, cited M3:<line>).

The reference main() calls, per step (M3:1285-1291),
    dt = compute_dt(p, U, B, dx, dy, dz)      (M3:626-648)
    rk2_step(p, U, B, dx, dy, dz, dt)         (M3:1034-1066)
on SoA std::vector<double> state Ucc {rho, mx, my, mz, E} and
Bfaces {Bx_f, By_f, Bz_f} (M3:91-99).  This module keeps those names and the
array layouts (cells (k*Ny+j)*Nx+i; faces with the face index along their own
axis running to N) and runs them through libcc_b200's C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _lib as L


@dataclass
class Params3:
    """Mirror of Params (M3:43-89), IC knobs omitted, plus the precision switch."""
    gamma1: float = 1.30
    gamma2: float = 2.50
    K1: float = 0.05
    rho_nuc: float = 80.0
    gamma_th: float = 1.50
    rho_bounce: float = 120.0
    gamma_bounce: float = 3.00
    Kbounce: float = 0.02
    gamma_init: float = 5.0 / 3.0
    cfl: float = 0.4
    x0: float = 0.0
    x1: float = 1.0
    y0: float = 0.0
    y1: float = 1.0
    z0: float = 0.0
    z1: float = 1.0
    Nx: int = 48
    Ny: int = 48
    Nz: int = 48
    t_end: float = 0.15
    dt_store: float = 1e-3
    floor_rho: float = 1e-10
    floor_P: float = 1e-10
    periodic_x: bool = True
    periodic_y: bool = True
    periodic_z: bool = True
    eta: float = 5e-4
    precision: str = "fp64"

    @staticmethod
    def ideal_gas(gamma: float = 5.0 / 3.0, **kw) -> "Params3":
        """The hybrid EOS reduced to an ideal gas of index gamma: no cold or
        bounce pressure (K1 = Kbounce = 0), thermal index gamma."""
        return Params3(K1=0.0, Kbounce=0.0, gamma_th=gamma, gamma_init=gamma, **kw)

    def to_c(self) -> L.CcMhd3dParams:
        c = L.CcMhd3dParams()
        for f in fields(self):
            if f.name == "precision":
                continue
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        c.precision = {"fp64": L.CC_FP64, "fp32": L.CC_FP32}[self.precision]
        return c

    @property
    def dx(self) -> float:
        return (self.x1 - self.x0) / self.Nx

    @property
    def dy(self) -> float:
        return (self.y1 - self.y0) / self.Ny

    @property
    def dz(self) -> float:
        return (self.z1 - self.z0) / self.Nz

    def sizes(self) -> list[int]:
        nx, ny, nz = self.Nx, self.Ny, self.Nz
        n = nx * ny * nz
        return [n] * 5 + [(nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)]


@dataclass
class State3:
    """Ucc {rho, mx, my, mz, E} and Bfaces {Bx_f, By_f, Bz_f} (M3:91-99)."""
    rho: np.ndarray
    mx: np.ndarray
    my: np.ndarray
    mz: np.ndarray
    E: np.ndarray
    Bx_f: np.ndarray
    By_f: np.ndarray
    Bz_f: np.ndarray

    def arrays(self) -> list[np.ndarray]:
        return [self.rho, self.mx, self.my, self.mz, self.E, self.Bx_f, self.By_f, self.Bz_f]

    def copy(self) -> "State3":
        return State3(*[a.copy() for a in self.arrays()])


def empty_state3(p: Params3) -> State3:
    return State3(*[np.zeros(n) for n in p.sizes()])
