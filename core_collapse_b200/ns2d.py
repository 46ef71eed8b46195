"""2D compressible Navier-Stokes + FFT self-gravity with first-order HLLC on
the GPU, behind the reference's own interface
(navier_stokes_2d_hllc_poisson.cpp, cited NS:<line>).

The reference main() calls, per step (NS:758-791),
    dt = compute_dt(U, g, p)          (NS:521-546), clamped to t_end
    compute_rhs(U, k1, g, p)          (NS:363-518), U1 = U + dt k1, rho floored
    compute_rhs(U1, k2, g, p)         U = U + dt/2 (k1 + k2), rho floored
on U4 {rho, rho u, rho v, E} (NS:88-90); every rhs solves the periodic
spectral Poisson problem of its own density (NS:379-383).  This module keeps
those names and the layout (q = i + Nx*j) and runs them through libcc_b200's
C ABI.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _lib as L

DERIVED_NS_FIELDS = ("rho", "P", "Mach", "u", "v", "momx", "momy", "Phi")


@dataclass
class ParamsNS:
    """Mirror of Params (NS:54-86), the HDF5 file name excepted."""
    gamma: float = 1.4
    cfl: float = 0.35
    x0: float = 0.0
    x1: float = 1.0
    y0: float = 0.0
    y1: float = 1.0
    Nx: int = 128
    Ny: int = 128
    t_end: float = 10.0
    dt_store: float = 5e-3
    seed: int = 42
    floor_rho: float = 1e-10
    floor_P: float = 1e-10
    viscosity_on: bool = True
    mu: float = 1e-6
    cfl_visc: float = 0.05
    gravity_on: bool = True
    G: float = 10.0
    precision: str = "fp64"

    def to_c(self) -> L.CcNs2dParams:
        c = L.CcNs2dParams()
        for f in fields(self):
            if f.name == "precision":
                continue
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        c.precision = {"fp64": L.CC_FP64, "fp32": L.CC_FP32}[self.precision]
        return c


@dataclass
class StateNS:
    """U4 {rho, mx, my, E} (NS:88-90), each Nx*Ny, q = i + Nx*j."""
    rho: np.ndarray
    mx: np.ndarray
    my: np.ndarray
    E: np.ndarray

    def arrays(self) -> list[np.ndarray]:
        return [self.rho, self.mx, self.my, self.E]

    def copy(self) -> "StateNS":
        return StateNS(*[a.copy() for a in self.arrays()])


def empty_state_ns(p: ParamsNS) -> StateNS:
    return StateNS(*[np.zeros(p.Nx * p.Ny) for _ in range(4)])


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "state arrays must be contiguous float64"
    return a.ctypes.data_as(L._DP)


def _ptrs(arrays):
    return (L._DP * len(arrays))(*[_dp(a) if a is not None else None for a in arrays])


class Ns2dSolver:
    """A device-resident 2D Navier-Stokes instance (one libcc_b200 handle)."""

    def __init__(self, p: ParamsNS):
        from .mhd2d import CcError
        self._Err = CcError
        self.p = p
        self._lib = L.lib()
        self._cp = p.to_c()
        self._h = C.c_void_p()
        self._t = 0.0
        r = self._lib.cc_ns2d_create(C.byref(self._cp), C.byref(self._h))
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

    def upload(self, s: StateNS):
        self._check(self._lib.cc_ns2d_upload(self._h, *[_dp(a) for a in s.arrays()]))
        self._t = 0.0

    def download(self, s: StateNS | None = None) -> StateNS:
        if s is None:
            s = empty_state_ns(self.p)
        self._check(self._lib.cc_ns2d_download(self._h, *[_dp(a) for a in s.arrays()]))
        return s

    def compute_dt(self) -> float:
        """compute_dt (NS:521-546) of the resident state."""
        dt = C.c_double()
        self._check(self._lib.cc_ns2d_compute_dt(self._h, C.byref(dt)))
        return dt.value

    def compute_gravity(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        """(phi, gx, gy) of the resident state (NS:285-360, 372-383)."""
        n = self.p.Nx * self.p.Ny
        phi, gx, gy = np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(self._lib.cc_ns2d_compute_gravity(self._h, _dp(phi), _dp(gx), _dp(gy)))
        return phi, gx, gy

    def compute_rhs(self) -> StateNS:
        """compute_rhs (NS:363-518) of the resident state."""
        d = empty_state_ns(self.p)
        self._check(self._lib.cc_ns2d_compute_rhs(self._h, _ptrs(d.arrays())))
        return d

    def rk2_step(self, dt: float):
        """One Heun step of the main() loop body (NS:762-781)."""
        self._check(self._lib.cc_ns2d_rk2_step(self._h, float(dt)))

    def advance(self, nsteps: int, t: float | None = None) -> float:
        """nsteps of the main loop from time t (None: where the last advance or
        upload (t = 0) left the clock); returns the time."""
        tt = C.c_double(self._t if t is None else t)
        self._check(self._lib.cc_ns2d_advance(self._h, int(nsteps), C.byref(tt)))
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
        """State, clock and parameters to one file (cc_ns2d_checkpoint_save)."""
        self._check(self._lib.cc_ns2d_checkpoint_save(self._h, str(path).encode()))

    def load_checkpoint(self, path: str):
        """Restore state and clock from a checkpoint of the same grid (cc_ns2d_checkpoint_load)."""
        self._check(self._lib.cc_ns2d_checkpoint_load(self._h, str(path).encode()))
        self._t = self.diagnostics()["t"]

    def diagnostics(self) -> dict:
        d = L.CcDiag()
        self._check(self._lib.cc_ns2d_diagnostics(self._h, C.byref(d)))
        return {f: getattr(d, f) for f, _ in L.CcDiag._fields_}

    def derived(self) -> dict:
        """The reference main()'s snapshot fields (NS:698-746), each (Ny, Nx)."""
        n = self.p.Nx * self.p.Ny
        out = [np.empty(n) for _ in DERIVED_NS_FIELDS]
        self._check(self._lib.cc_ns2d_derived(self._h, _ptrs(out)))
        return {k: a.reshape(self.p.Ny, self.p.Nx) for k, a in zip(DERIVED_NS_FIELDS, out)}


def compute_rhs(p: ParamsNS, U: StateNS) -> StateNS:
    """compute_rhs (NS:363-518) on the GPU."""
    with Ns2dSolver(p) as g:
        g.upload(U)
        return g.compute_rhs()


def compute_dt(p: ParamsNS, U: StateNS) -> float:
    """compute_dt (NS:521-546) on the GPU."""
    with Ns2dSolver(p) as g:
        g.upload(U)
        return g.compute_dt()


def ic_collapse(p: ParamsNS) -> StateNS:
    """The reference main()'s collapse IC (NS:627-689)."""
    U = empty_state_ns(p)
    cp = p.to_c()
    if L.lib().cc_ic_ns2d_collapse(C.byref(cp), _ptrs(U.arrays())) != 0:
        raise ValueError("cc_ic_ns2d_collapse failed")
    return U
