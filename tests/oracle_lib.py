"""Test-side access to the CPU checkers under oracle/ (never used by the
product): liboracle.so (the restatement) and oracle/_ref/libref_*.so (the
reference solvers compiled in place).  Built by `make -C oracle`."""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

from core_collapse_b200 import _lib as L

ROOT = Path(__file__).resolve().parents[1]
ORACLE_DIR = ROOT / "oracle"
REF_DIR = ORACLE_DIR / "_ref"
# the reference tree: $CC_REFERENCE_DIR, else a checkout named `reference` beside this repository
REFERENCE_SRC = Path(os.environ.get("CC_REFERENCE_DIR") or ROOT.parent / "reference")

_DP = C.POINTER(C.c_double)
_PP = C.POINTER(_DP)


def build_oracle():
    """(Re)build liboracle.so and, where the reference tree exists, _ref/*.so."""
    subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True, capture_output=True)


def _load(path: Path) -> C.CDLL | None:
    return C.CDLL(str(path)) if path.exists() else None


_oracle = None
_refs: dict = {}


def oracle() -> C.CDLL:
    global _oracle
    if _oracle is None:
        if not (ORACLE_DIR / "liboracle.so").exists():
            build_oracle()
        O = C.CDLL(str(ORACLE_DIR / "liboracle.so"))
        P2 = C.POINTER(L.CcMhd2dParams)
        O.or_mhd2d_gravity.argtypes = [P2, _DP, _DP, _DP, C.c_int, C.POINTER(C.c_int), _DP]
        O.or_mhd2d_phi.argtypes = [P2, _DP, _DP, C.c_int, C.POINTER(C.c_int), _DP]
        O.or_mhd2d_compute_dt.argtypes = [P2, _PP]
        O.or_mhd2d_compute_dt.restype = C.c_double
        O.or_mhd2d_advance_stage.argtypes = [P2, _PP, _PP, _DP, _DP, C.c_double]
        O.or_mhd2d_rk2_step.argtypes = [P2, _PP, _DP, _DP, C.c_double, C.c_int]
        O.or_mhd2d_main_loop.argtypes = [P2, _PP, C.c_int, _DP, C.c_int, C.c_int]
        O.or_mhd2d_divB_max.argtypes = [P2, _PP]
        O.or_mhd2d_divB_max.restype = C.c_double
        O.or_mhd2d_derived.argtypes = [P2, _PP, _PP]
        O.or_mhd2d_derived.restype = None
        O.or_fft1d.argtypes = [C.c_int, _DP, C.c_int]
        PE = C.POINTER(L.CcEuler2dParams)
        O.or_euler2d_gravity.argtypes = [PE, _DP, _DP, _DP, C.c_int, C.POINTER(C.c_int), _DP]
        O.or_euler2d_rhs.argtypes = [PE, _PP, _PP, C.c_int]
        O.or_euler2d_compute_dt.argtypes = [PE, _PP]
        O.or_euler2d_compute_dt.restype = C.c_double
        O.or_euler2d_derived.argtypes = [PE, _PP, _PP]
        O.or_euler2d_derived.restype = None
        O.or_euler2d_rk2_step.argtypes = [PE, _PP, C.c_double, C.c_int]
        O.or_euler2d_main_loop.argtypes = [PE, _PP, C.c_int, _DP, C.c_int, C.c_int]
        PN = C.POINTER(L.CcNs2dParams)
        O.or_ns2d_ic.argtypes = [PN, _PP]
        O.or_ns2d_gravity.argtypes = [PN, _PP, _DP, _DP, _DP]
        O.or_ns2d_rhs.argtypes = [PN, _PP, _PP]
        O.or_ns2d_compute_dt.argtypes = [PN, _PP]
        O.or_ns2d_compute_dt.restype = C.c_double
        O.or_ns2d_rk2_step.argtypes = [PN, _PP, C.c_double]
        O.or_ns2d_derived.argtypes = [PN, _PP, _PP]
        O.or_ns2d_derived.restype = None
        O.or_ns2d_main_loop.argtypes = [PN, _PP, C.c_int, _DP, C.c_int]
        P3 = C.POINTER(L.CcMhd3dParams)
        O.or_mhd3d_advance_stage.argtypes = [P3, _PP, _PP, C.c_double]
        O.or_mhd3d_rk2_step.argtypes = [P3, _PP, C.c_double]
        O.or_mhd3d_compute_dt.argtypes = [P3, _PP]
        O.or_mhd3d_compute_dt.restype = C.c_double
        O.or_mhd3d_main_loop.argtypes = [P3, _PP, C.c_int, _DP, C.c_int]
        O.or_mhd3d_divB_max.argtypes = [P3, _PP]
        O.or_mhd3d_divB_max.restype = C.c_double
        O.or_mhd3d_derived.argtypes = [P3, _PP, _PP]
        O.or_mhd3d_derived.restype = None
        O.or_mhd2d_tlm.argtypes = [C.POINTER(L.CcMhd2dParams), _PP, _PP, C.c_int, _DP]
        O.or_poisson_generic.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.c_double, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, _DP, _DP,
                                         _DP, C.POINTER(C.c_int), _DP]
        _oracle = O
    return _oracle


def ref(name: str) -> C.CDLL | None:
    """The reference solver library `name` in {mhd2d, mhd3d, euler2d, fft, ge}, or None."""
    if name not in _refs:
        path = REF_DIR / f"libref_{name}.so"
        if not path.exists() and REFERENCE_SRC.exists():
            build_oracle()
        R = _load(path)
        if R is not None and name == "mhd2d":
            P2 = C.POINTER(L.CcMhd2dParams)
            R.ref_mhd2d_rk2_step.argtypes = [P2, _PP, _DP, _DP, C.c_double]
            R.ref_mhd2d_advance_stage.argtypes = [P2, _PP, _PP, _DP, _DP, C.c_double]
            R.ref_mhd2d_compute_dt.argtypes = [P2, _PP]
            R.ref_mhd2d_compute_dt.restype = C.c_double
            R.ref_mhd2d_poisson.argtypes = [P2, _DP, _DP, _DP]
            R.ref_mhd2d_main_loop.argtypes = [P2, _PP, C.c_int, _DP]
            R.ref_mhd2d_divB_max.argtypes = [P2, _PP]
            R.ref_mhd2d_divB_max.restype = C.c_double
        if R is not None and name == "mhd3d":
            P3 = C.POINTER(L.CcMhd3dParams)
            R.ref_mhd3d_rk2_step.argtypes = [P3, _PP, C.c_double]
            R.ref_mhd3d_advance_stage.argtypes = [P3, _PP, _PP, C.c_double]
            R.ref_mhd3d_compute_dt.argtypes = [P3, _PP]
            R.ref_mhd3d_compute_dt.restype = C.c_double
            R.ref_mhd3d_main_loop.argtypes = [P3, _PP, C.c_int, _DP]
            R.ref_mhd3d_divB_max.argtypes = [P3, _PP]
            R.ref_mhd3d_divB_max.restype = C.c_double
        if R is not None and name == "euler2d":
            P2 = C.POINTER(L.CcEuler2dParams)
            R.ref_euler2d_rk2_step.argtypes = [P2, _PP, C.c_double]
            R.ref_euler2d_rhs.argtypes = [P2, _PP, _PP]
            R.ref_euler2d_compute_dt.argtypes = [P2, _PP]
            R.ref_euler2d_compute_dt.restype = C.c_double
            R.ref_euler2d_poisson.argtypes = [P2, _PP, _DP, _DP]
            R.ref_euler2d_enclosed_gravity.argtypes = [P2, _PP, _DP, _DP]
            R.ref_euler2d_init_random_blob.argtypes = [P2, _PP]
            R.ref_euler2d_main_loop.argtypes = [P2, _PP, C.c_int, _DP]
        if R is not None and name == "ge":
            R.ref_ge_gravity.argtypes = [C.c_int, C.c_int] + [C.c_double] * 6 + [C.c_int] + [C.c_double] * 3 + \
                [_DP, _DP, _DP]
        if R is not None and name == "fft":
            R.ref_fft_poisson.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                          C.c_double, _DP, _DP]
            R.ref_fft_gravity_accel.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                                _DP, _DP, _DP]
            R.ref_fft1d.argtypes = [C.c_int, _DP, C.c_int]
            R.ref_ns_rhs.argtypes = [C.c_int, C.c_int] + [C.c_double] * 7 + [C.c_int, C.c_double, C.c_int,
                                                                             C.c_double, _PP, _PP]
            R.ref_ns_dt.argtypes = [C.c_int, C.c_int] + [C.c_double] * 8 + [C.c_int, C.c_double, C.c_double, _PP]
            R.ref_ns_dt.restype = C.c_double
        _refs[name] = R
    return _refs[name]


def dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_DP)


def pp(arrays) -> C.Array:
    """Pointer array over `arrays`; it holds references to them, so a
    temporary list stays alive for as long as the pointer array does."""
    arrays = list(arrays)
    out = (_DP * len(arrays))(*[dp(a) for a in arrays])
    out._keep = arrays
    return out


# ---- state helpers: a 2D MHD state is the list [rho, mx, my, mz, E, Bz, Bx_f, By_f] ----

def state_list(U, B) -> list[np.ndarray]:
    return [a.copy() for a in U.arrays()] + [B.Bx_f.copy(), B.By_f.copy()]


def copy_state(S):
    return [a.copy() for a in S]


def m2_rk2_ref(cp, S, gx, gy, dt):
    out = copy_state(S)
    ref("mhd2d").ref_mhd2d_rk2_step(C.byref(cp), pp(out), dp(gx), dp(gy), dt)
    return out


def m2_rk2_oracle(cp, S, gx, gy, dt, mode):
    out = copy_state(S)
    oracle().or_mhd2d_rk2_step(C.byref(cp), pp(out), dp(gx), dp(gy), dt, mode)
    return out


def m2_stage_ref(cp, S, gx, gy, dt):
    out = [np.zeros_like(a) for a in S]
    ref("mhd2d").ref_mhd2d_advance_stage(C.byref(cp), pp(S), pp(out), dp(gx), dp(gy), dt)
    return out


def m2_stage_oracle(cp, S, gx, gy, dt):
    out = [np.zeros_like(a) for a in S]
    oracle().or_mhd2d_advance_stage(C.byref(cp), pp(S), pp(out), dp(gx), dp(gy), dt)
    return out


def m2_gravity_oracle(cp, rho, mode):
    n = cp.Nx * cp.Ny
    gx, gy = np.zeros(n), np.zeros(n)
    it = C.c_int()
    res = C.c_double()
    oracle().or_mhd2d_gravity(C.byref(cp), dp(np.ascontiguousarray(rho)), dp(gx), dp(gy), mode, C.byref(it),
                              C.byref(res))
    return gx, gy, it.value, res.value


def m2_main_loop_oracle(cp, S, nsteps, mode, fp32=False, t0=0.0):
    out = copy_state(S)
    t = C.c_double(t0)
    oracle().or_mhd2d_main_loop(C.byref(cp), pp(out), nsteps, C.byref(t), mode, 1 if fp32 else 0)
    return out, t.value


def m2_derived_oracle(cp, S) -> list[np.ndarray]:
    """The reference main()'s snapshot fields (rho, P, Mach, u, v, vabs, Bx,
    By, Bz, divB) of state S, restated on the CPU."""
    n = cp.Nx * cp.Ny
    out = [np.empty(n) for _ in range(10)]
    oracle().or_mhd2d_derived(C.byref(cp), pp(S), pp(out))
    return out


def rel_linf(a: np.ndarray, b: np.ndarray) -> float:
    """max|a-b| / max|b| (0 when both are identically zero)."""
    den = float(np.max(np.abs(b))) if b.size else 0.0
    num = float(np.max(np.abs(a - b))) if a.size else 0.0
    if den == 0.0:
        return num
    return num / den


# ---- 3D state helpers: [rho, mx, my, mz, E, Bx_f, By_f, Bz_f] ----

def m3_rk2_ref(cp, S, dt):
    out = copy_state(S)
    ref("mhd3d").ref_mhd3d_rk2_step(C.byref(cp), pp(out), dt)
    return out


def m3_rk2_oracle(cp, S, dt):
    out = copy_state(S)
    oracle().or_mhd3d_rk2_step(C.byref(cp), pp(out), dt)
    return out


def m3_main_loop_oracle(cp, S, nsteps, fp32=False, t0=0.0):
    out = copy_state(S)
    t = C.c_double(t0)
    oracle().or_mhd3d_main_loop(C.byref(cp), pp(out), nsteps, C.byref(t), 1 if fp32 else 0)
    return out, t.value


# ---- 2D Euler helpers: [rho, mx, my, E] ----

def eh_main_loop_oracle(cp, S, nsteps, mode, fp32=False, t0=0.0):
    out = copy_state(S)
    t = C.c_double(t0)
    rc = oracle().or_euler2d_main_loop(C.byref(cp), pp(out), nsteps, C.byref(t), mode, 1 if fp32 else 0)
    return out, t.value, rc


# ---- 2D Navier-Stokes helpers: [rho, mx, my, E] ----

def ns_main_loop_oracle(cp, S, nsteps, fp32=False, t0=0.0):
    out = copy_state(S)
    t = C.c_double(t0)
    oracle().or_ns2d_main_loop(C.byref(cp), pp(out), nsteps, C.byref(t), 1 if fp32 else 0)
    return out, t.value


def ns_rhs_oracle(cp, S):
    out = [np.zeros_like(a) for a in S]
    oracle().or_ns2d_rhs(C.byref(cp), pp(S), pp(out))
    return out


def ns_ref_rhs(cp, S):
    """compute_rhs of the compiled reference (None without it)."""
    R = ref("fft")
    if R is None:
        return None
    out = [np.zeros_like(a) for a in S]
    R.ref_ns_rhs(cp.Nx, cp.Ny, cp.x0, cp.x1, cp.y0, cp.y1, cp.gamma, cp.floor_rho, cp.floor_P, cp.viscosity_on,
                 cp.mu, cp.gravity_on, cp.G, pp(S), pp(out))
    return out


def ns_ref_dt(cp, S):
    R = ref("fft")
    if R is None:
        return None
    return R.ref_ns_dt(cp.Nx, cp.Ny, cp.x0, cp.x1, cp.y0, cp.y1, cp.gamma, cp.cfl, cp.floor_rho, cp.floor_P,
                       cp.viscosity_on, cp.mu, cp.cfl_visc, pp(S))
