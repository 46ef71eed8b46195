"""The 3D reference initial condition (cc_ic_mhd3d_reference,
mhd3d_resistive_hlld_ct.cpp:1159-1272), host code: checked on the CPU."""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle_lib as O
from core_collapse_b200.mhd3d import Params3, ic_reference3


def test_ic3d_reference_fields():
    p = Params3(Nx=12, Ny=10, Nz=8)
    s = ic_reference3(p)
    cp = p.to_c()
    # divergence-free faces (curl of the corner potential plus uniform fields)
    assert O.oracle().or_mhd3d_divB_max(C.byref(cp), O.pp([a.copy() for a in s.arrays()])) < 1e-12
    assert np.all(s.Bz_f == 0.05)
    # density and momentum of the tanh core with infall and rotation (M3:1228-1262)
    x = p.x0 + (np.arange(p.Nx) + 0.5) * (p.x1 - p.x0) / p.Nx
    y = p.y0 + (np.arange(p.Ny) + 0.5) * (p.y1 - p.y0) / p.Ny
    z = p.z0 + (np.arange(p.Nz) + 0.5) * (p.z1 - p.z0) / p.Nz
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rx, ry, rz = X - 0.5, Y - 0.5, Z - 0.5
    r = np.sqrt(rx * rx + ry * ry + rz * rz) + 1e-14
    core = 0.5 * (1.0 - np.tanh((r - 0.12) / 0.02))
    rho = 1.0 + (20.0 - 1.0) * core
    u = -1.25 * core * rx / r - 1.0 * (Y - 0.5)
    assert np.allclose(s.rho.reshape(rho.shape), rho, rtol=1e-14, atol=0)
    assert np.allclose(s.mx.reshape(rho.shape), rho * u, rtol=1e-12, atol=1e-14)
    assert np.all(np.isfinite(s.E)) and np.all(s.E > 0)


def test_ic3d_rejects_null():
    from core_collapse_b200 import _lib as L
    p = Params3(Nx=4, Ny=4, Nz=4)
    cp = p.to_c()
    arr = (C.POINTER(C.c_double) * 8)()
    assert L.lib().cc_ic_mhd3d_reference(C.byref(cp), None, arr) == -1
