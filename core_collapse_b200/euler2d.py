"""2D Euler + self-gravity with HLLC on the GPU, behind the reference's own
interface (euler2d_gravity_hllc.cpp, cited EH:<line>).

The reference main() calls, per step (EH:697-706),
    dt = compute_dt(p, U)          (EH:390-404), aborting on a non-finite or non-positive dt
    rk2_step(p, U, dt)             (EH:529-550), whose rhs solves Poisson itself (EH:411)
on State {rho, mx, my, E} (EH:58-60).  This module keeps those names and the
layouts (q = j*Nx + i) and runs them through libcc_b200's C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _lib as L


@dataclass
class ParamsEH:
    """Mirror of Params (EH:29-56); the SOR constants the reference hard-codes
    inside its Poisson solve (EH:329-331) are fields here."""
    gamma: float = 1.2
    cfl: float = 0.45
    x0: float = 0.0
    x1: float = 1.0
    y0: float = 0.0
    y1: float = 1.0
    Nx: int = 50
    Ny: int = 50
    t_end: float = 5.0
    dt_store: float = 1e-3
    floor_rho: float = 1e-12
    floor_P: float = 1e-12
    periodic_x: bool = True
    periodic_y: bool = True
    gravity_on: bool = True
    sor_max_iter: int = 50000
    G: float = 1.0
    softening: float = 1e-4
    sor_tol: float = 1e-10
    sor_omega: float = 1.7
    poisson: str = "sor"       # "sor": red-black SOR; "sor_lex": the reference's lexicographic SOR
    #                            (a parity mode); "enclosed": enclosed-mass radial gravity (EH:226-286);
    #                            "shells": shell-binned enclosed mass (gravity_enclosed.h:18-96)
    precision: str = "fp64"
    Nr_bins: int = 512         # shell count of "shells" (euler2d_h5.cpp:43)
    xc: float = 0.5            # gravity centre of "shells" (euler2d_h5.cpp:44-45)
    yc: float = 0.5

    def to_c(self) -> L.CcEuler2dParams:
        c = L.CcEuler2dParams()
        for f in fields(self):
            if f.name in ("poisson", "precision"):
                continue
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        c.poisson_kind = {"sor": L.CC_POISSON_SOR, "fft": L.CC_POISSON_FFT, "sor_lex": L.CC_POISSON_SOR_LEX,
                          "enclosed": L.CC_GRAVITY_ENCLOSED, "shells": L.CC_GRAVITY_SHELLS}[self.poisson]
        c.precision = {"fp64": L.CC_FP64, "fp32": L.CC_FP32}[self.precision]
        return c

    @property
    def dx(self) -> float:
        return (self.x1 - self.x0) / self.Nx

    @property
    def dy(self) -> float:
        return (self.y1 - self.y0) / self.Ny


@dataclass
class StateEH:
    """State {rho, mx, my, E} (EH:58-60), each Nx*Ny."""
    rho: np.ndarray
    mx: np.ndarray
    my: np.ndarray
    E: np.ndarray

    def arrays(self) -> list[np.ndarray]:
        return [self.rho, self.mx, self.my, self.E]

    def copy(self) -> "StateEH":
        return StateEH(*[a.copy() for a in self.arrays()])


def empty_state_eh(p: ParamsEH) -> StateEH:
    return StateEH(*[np.zeros(p.Nx * p.Ny) for _ in range(4)])


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "state arrays must be contiguous float64"
    return a.ctypes.data_as(L._DP)


class Euler2dSolver:
    """A device-resident 2D Euler/HLLC instance (one libcc_b200 handle)."""

    def __init__(self, p: ParamsEH):
        from .mhd2d import CcError
        self._Err = CcError
        self.p = p
        self._lib = L.lib()
        self._cp = p.to_c()
        self._h = C.c_void_p()
        r = self._lib.cc_euler2d_create(C.byref(self._cp), C.byref(self._h))
        if r != L.CC_OK:
            msg = self._lib.cc_last_error(self._h).decode() if self._h.value else "create failed"
            if self._h.value:
                self._lib.cc_destroy(self._h)
            self._h = C.c_void_p()
            raise CcError(r, msg)

    def _check(self, r: int):
        if r != L.CC_OK:
            raise self._Err(r, self._lib.cc_last_error(self._h).decode())

    def close(self):
        if self._h and self._h.value:
            self._lib.cc_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def upload(self, s: StateEH):
        self._check(self._lib.cc_euler2d_upload(self._h, *[_dp(a) for a in s.arrays()]))
        self._t = 0.0

    def download(self, s: StateEH | None = None) -> StateEH:
        if s is None:
            s = empty_state_eh(self.p)
        self._check(self._lib.cc_euler2d_download(self._h, *[_dp(a) for a in s.arrays()]))
        return s

    def compute_dt(self) -> float:
        dt = C.c_double()
        self._check(self._lib.cc_euler2d_compute_dt(self._h, C.byref(dt)))
        return dt.value

    def compute_gravity(self) -> tuple[np.ndarray, np.ndarray]:
        n = self.p.Nx * self.p.Ny
        gx, gy = np.zeros(n), np.zeros(n)
        self._check(self._lib.cc_euler2d_compute_gravity(self._h, _dp(gx), _dp(gy)))
        return gx, gy

    def rk2_step(self, dt: float):
        self._check(self._lib.cc_euler2d_rk2_step(self._h, float(dt)))

    def advance(self, nsteps: int, t: float | None = None) -> float:
        """nsteps of the main loop from time t (None: where the last advance or
        upload (t = 0) left the clock); returns the time."""
        tt = C.c_double(getattr(self, "_t", 0.0) if t is None else t)
        self._check(self._lib.cc_euler2d_advance(self._h, int(nsteps), C.byref(tt)))
        self._t = tt.value
        return tt.value

    def set_stream(self, stream_ptr: int | None):
        """Queue this handle's work on a caller's cudaStream_t (None: its own stream)."""
        self._check(self._lib.cc_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def perf(self) -> dict:
        q = L.CcPerf()
        self._check(self._lib.cc_get_perf(self._h, C.byref(q)))
        return {f: getattr(q, f) for f, _ in L.CcPerf._fields_}

    def reset_perf(self):
        self._check(self._lib.cc_reset_perf(self._h))

    def save_checkpoint(self, path: str):
        """State, clock and parameters to one file (cc_euler2d_checkpoint_save)."""
        self._check(self._lib.cc_euler2d_checkpoint_save(self._h, str(path).encode()))

    def load_checkpoint(self, path: str):
        """Restore state and clock from a checkpoint of the same grid (cc_euler2d_checkpoint_load)."""
        self._check(self._lib.cc_euler2d_checkpoint_load(self._h, str(path).encode()))
        self._t = self.diagnostics()["t"]

    def diagnostics(self) -> dict:
        d = L.CcDiag()
        self._check(self._lib.cc_euler2d_diagnostics(self._h, C.byref(d)))
        return {f: getattr(d, f) for f, _ in L.CcDiag._fields_}

    def derived(self) -> dict:
        """The reference main()'s snapshot fields (EH:661-689): {rho, P, Mach}, each (Ny, Nx)."""
        n = self.p.Nx * self.p.Ny
        out = [np.empty(n) for _ in range(3)]
        arr = (C.POINTER(C.c_double) * 3)(*[a.ctypes.data_as(L._DP) for a in out])
        self._check(self._lib.cc_euler2d_derived(self._h, arr))
        return {k: a.reshape(self.p.Ny, self.p.Nx) for k, a in zip(("rho", "P", "Mach"), out)}


def compute_dt(p: ParamsEH, U: StateEH) -> float:
    """compute_dt (EH:390-404) on the GPU."""
    with Euler2dSolver(p) as g:
        g.upload(U)
        return g.compute_dt()


def rk2_step(p: ParamsEH, U: StateEH, dt: float) -> None:
    """rk2_step (EH:529-550) on the GPU; U is updated in place."""
    with Euler2dSolver(p) as g:
        g.upload(U)
        g.rk2_step(dt)
        g.download(U)


def ic_random_blob(p: ParamsEH) -> StateEH:
    """The reference main()'s IC, init_random_blob (EH:574-642)."""
    U = empty_state_eh(p)
    cp = p.to_c()
    arr = (L._DP * 4)(*[_dp(a) for a in U.arrays()])
    if L.lib().cc_ic_euler2d_random_blob(C.byref(cp), arr) != 0:
        raise ValueError("cc_ic_euler2d_random_blob failed")
    return U
