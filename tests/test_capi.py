"""libcc_b200.so loads without a GPU and exports every function that
include/*.h declares; host-only entry points (defaults, initial conditions)
behave; argument errors are reported, not crashed on."""
import ctypes as C
import re
from pathlib import Path

import numpy as np

from core_collapse_b200 import _lib as L
from core_collapse_b200.mhd2d import Params, ic_collapse, ic_orszag_tang, ic_reference

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_functions() -> set[str]:
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(cc_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 15
    lib = C.CDLL(str(L.LIB_PATH))
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, f"declared but not exported: {missing}"
    # and the Python binding knows every one of them
    assert not (names - set(L.SIGNATURES)), f"not bound in _lib.SIGNATURES: {names - set(L.SIGNATURES)}"


def test_params_struct_layout_matches_defaults():
    p = L.CcMhd2dParams()
    L.lib().cc_mhd2d_params_default(C.byref(p))
    # M2:44-72 defaults
    assert p.gamma == 5.0 / 3.0 and p.cfl == 0.45 and p.Nx == 192 and p.Ny == 192
    assert p.t_end == 0.35 and p.floor_rho == 1e-10 and p.periodic_x == 1 and p.eta == 5e-4
    assert p.gravity_on == 1 and p.G == 8.0 and p.sor_iters == 600 and p.sor_omega == 1.8
    assert C.sizeof(L.CcMhd2dParams) == 168


def test_create_rejects_bad_arguments_without_gpu_work():
    lib = L.lib()
    h = C.c_void_p()
    bad = Params(Nx=1).to_c()
    assert lib.cc_mhd2d_create(C.byref(bad), C.byref(h)) == L.CC_ERR_ARG
    assert lib.cc_mhd2d_create(None, C.byref(h)) == L.CC_ERR_ARG
    assert lib.cc_destroy(None) == L.CC_ERR_ARG
    assert lib.cc_last_error(None) == b"null handle"


def test_batch_create_validates_instances_before_gpu_work():
    """cc_batch_create checks every instance before touching the device; the
    message names the instance."""
    lib = L.lib()
    ok = Params(Nx=16, Ny=16, gravity_on=True, poisson="direct")
    cases = [
        ([ok, Params(Nx=16, Ny=16, gravity_on=True, poisson="sor")], L.CC_ERR_UNSUPPORTED, b"instance 1"),
        ([ok, Params(Nx=3, Ny=16, gravity_on=False)], L.CC_ERR_ARG, b"instance 1"),
        ([Params(Nx=16, Ny=16, precision="fp32", gravity_on=False), ok], L.CC_ERR_ARG, b"one precision"),
        ([Params(Nx=4096, Ny=16, gravity_on=True, poisson="direct")], L.CC_ERR_UNSUPPORTED, b"instance 0"),
    ]
    for plist, code, msg in cases:
        arr = (L.CcMhd2dParams * len(plist))(*[q.to_c() for q in plist])
        h = C.c_void_p()
        assert lib.cc_batch_create(arr, len(plist), C.byref(h)) == code
        assert msg in lib.cc_last_error(h)
        assert lib.cc_destroy(h) == L.CC_OK
    h = C.c_void_p()
    assert lib.cc_batch_create(None, 1, C.byref(h)) == L.CC_ERR_ARG
    assert lib.cc_batch_advance(None, 1, None) == L.CC_ERR_ARG


def test_ic_collapse_is_seeded_and_divergence_free():
    p = Params(Nx=32, Ny=24, x0=-1, x1=1, y0=-1, y1=1, periodic_x=False, periodic_y=False)
    U1, B1 = ic_collapse(p, seed=0)
    U2, B2 = ic_collapse(p, seed=0)
    U3, _ = ic_collapse(p, seed=1)
    assert np.array_equal(U1.rho, U2.rho) and not np.array_equal(U1.rho, U3.rho)
    assert U1.rho.max() > 8.0 and U1.rho.min() > 0.98
    assert np.all(B1.Bx_f == 0.05) and np.all(B1.By_f == 0.0)
    # P = 0.1 rho^(5/3) recovered from E (no kinetic or Bz energy)
    P = (p.gamma - 1) * (U1.E - 0.5 * 0.05 ** 2)
    assert np.allclose(P, 0.1 * U1.rho ** (5 / 3), rtol=1e-12)


def _divB(p, B):
    bx = B.Bx_f.reshape(p.Ny, p.Nx + 1)
    by = B.By_f.reshape(p.Ny + 1, p.Nx)
    return (bx[:, 1:] - bx[:, :-1]) / p.dx + (by[1:, :] - by[:-1, :]) / p.dy


def test_ic_orszag_tang_fields():
    p = Params(Nx=64, Ny=64, x0=-1, x1=1, y0=-1, y1=1)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.1)
    assert np.max(np.abs(_divB(p, B))) < 1e-12
    x = p.x0 + (np.arange(p.Nx) + 0.5) * p.dx
    y = p.y0 + (np.arange(p.Ny) + 0.5) * p.dy
    X, Y = np.meshgrid(x, y)
    rho = 25 / (36 * np.pi) + 4.0 * np.exp(-(X ** 2 + Y ** 2) / (2 * 0.1 ** 2))
    assert np.allclose(U.rho.reshape(p.Ny, p.Nx), rho, rtol=1e-14)
    assert np.allclose(U.mx.reshape(p.Ny, p.Nx), -rho * np.sin(2 * np.pi * Y), atol=1e-14)


def test_ic_reference_divergence_free():
    p = Params(Nx=48, Ny=40)
    U, B = ic_reference(p)
    assert np.max(np.abs(_divB(p, B))) < 1e-10
    assert U.rho.max() > 19.0 and U.rho.min() >= 1.0 - 1e-12
