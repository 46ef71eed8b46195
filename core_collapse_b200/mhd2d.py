"""2D resistive MHD + self-gravity on the GPU, behind the reference's own
interface (mhd2d_resistive_hlld_ct_gravity.cpp, cited M2:<line>).

The reference is one C++ translation unit whose main() calls
    compute_poisson_gravity_periodic(p, U.rho, dx, dy) -> GravField   (M2:178)
    compute_dt(p, U, B, dx, dy) -> double                             (M2:579)
    rk2_step(p, U, B, g, dx, dy, dt)                                  (M2:838)
on SoA std::vector<double> state (Ucc, Bfaces, GravField: M2:88-99).  This
module keeps those names, arguments and in-place semantics, with numpy
arrays in the reference layouts, and runs them through libcc_b200's C ABI.
`Mhd2dSolver` keeps the state resident on the device for time loops.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields

import numpy as np

from . import _lib as L


@dataclass
class Params:
    """Mirror of Params (M2:44-86) plus the step options this library adds."""
    gamma: float = 5.0 / 3.0
    cfl: float = 0.45
    x0: float = 0.0
    x1: float = 1.0
    y0: float = 0.0
    y1: float = 1.0
    Nx: int = 192
    Ny: int = 192
    t_end: float = 0.35
    dt_store: float = 1e-3
    floor_rho: float = 1e-10
    floor_P: float = 1e-10
    periodic_x: bool = True
    periodic_y: bool = True
    eta: float = 5e-4
    gravity_on: bool = True
    G: float = 8.0
    softening: float = 1e-4
    sor_iters: int = 600
    sor_omega: float = 1.8
    # additions
    sor_tol: float = 0.0            # > 0: stop SOR once max|lap(phi)-rhs| < sor_tol
    poisson: str = "sor"            # "sor" (red-black), "fft", "sor_lex" (the reference's lexicographic
    #                                 SOR, a parity mode) or "direct" (batched ensemble only)
    precision: str = "fp64"         # "fp64" or "fp32"
    compensated: bool = False       # FP32 only: compensated (Kahan-style) state update

    def to_c(self) -> L.CcMhd2dParams:
        c = L.CcMhd2dParams()
        for f in fields(self):
            if f.name in ("poisson", "precision"):
                continue
            v = getattr(self, f.name)
            setattr(c, f.name, int(v) if isinstance(v, bool) else v)
        c.poisson_kind = {"sor": L.CC_POISSON_SOR, "fft": L.CC_POISSON_FFT, "direct": L.CC_POISSON_DIRECT,
                          "sor_lex": L.CC_POISSON_SOR_LEX}[self.poisson]
        c.precision = {"fp64": L.CC_FP64, "fp32": L.CC_FP32}[self.precision]
        return c

    @property
    def dx(self) -> float:
        return (self.x1 - self.x0) / self.Nx

    @property
    def dy(self) -> float:
        return (self.y1 - self.y0) / self.Ny


@dataclass
class Ucc:
    """Cell-centred conserved state (M2:88-90), each Nx*Ny, q = j*Nx + i."""
    rho: np.ndarray
    mx: np.ndarray
    my: np.ndarray
    mz: np.ndarray
    E: np.ndarray
    Bz: np.ndarray

    def arrays(self):
        return [self.rho, self.mx, self.my, self.mz, self.E, self.Bz]

    def copy(self) -> "Ucc":
        return Ucc(*[a.copy() for a in self.arrays()])


@dataclass
class Bfaces:
    """Face-centred in-plane B (M2:92-95): Bx_f (Nx+1)*Ny, By_f Nx*(Ny+1)."""
    Bx_f: np.ndarray
    By_f: np.ndarray

    def copy(self) -> "Bfaces":
        return Bfaces(self.Bx_f.copy(), self.By_f.copy())


@dataclass
class GravField:
    """Cell-centred gravitational acceleration (M2:97-99)."""
    gx: np.ndarray
    gy: np.ndarray


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "state arrays must be contiguous float64"
    return a.ctypes.data_as(L._DP)


def empty_state(p: Params) -> tuple[Ucc, Bfaces]:
    n = p.Nx * p.Ny
    U = Ucc(*[np.zeros(n) for _ in range(6)])
    B = Bfaces(np.zeros((p.Nx + 1) * p.Ny), np.zeros(p.Nx * (p.Ny + 1)))
    return U, B


def _state_ptrs(U: Ucc, B: Bfaces):
    return [_dp(a) for a in U.arrays()] + [_dp(B.Bx_f), _dp(B.By_f)]


class CcError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cc error {code}: {msg}")
        self.code = code


# output order of the reference's snapshot store (M2:1090-1104, written by write_h5)
DERIVED_FIELDS = ("rho", "P", "Mach", "u", "v", "vabs", "Bx", "By", "Bz", "divB")


class Mhd2dSolver:
    """A device-resident 2D MHD instance (one libcc_b200 handle)."""

    def __init__(self, p: Params):
        self.p = p
        self._lib = L.lib()
        self._cp = p.to_c()
        self._h = C.c_void_p()
        r = self._lib.cc_mhd2d_create(C.byref(self._cp), C.byref(self._h))
        if r != L.CC_OK:
            msg = self._lib.cc_last_error(self._h).decode() if self._h.value else "create failed"
            if self._h.value:
                self._lib.cc_destroy(self._h)
            self._h = C.c_void_p()
            raise CcError(r, msg)

    def _check(self, r: int):
        if r != L.CC_OK:
            raise CcError(r, self._lib.cc_last_error(self._h).decode())

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

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def upload(self, U: Ucc, B: Bfaces):
        self._check(self._lib.cc_mhd2d_upload(self._h, *_state_ptrs(U, B)))
        self._t = 0.0

    def download(self, U: Ucc | None = None, B: Bfaces | None = None) -> tuple[Ucc, Bfaces]:
        if U is None or B is None:
            U, B = empty_state(self.p)
        self._check(self._lib.cc_mhd2d_download(self._h, *_state_ptrs(U, B)))
        return U, B

    def compute_gravity(self, to_host: bool = True) -> GravField | None:
        if to_host:
            n = self.p.Nx * self.p.Ny
            g = GravField(np.zeros(n), np.zeros(n))
            self._check(self._lib.cc_mhd2d_compute_gravity(self._h, _dp(g.gx), _dp(g.gy)))
            return g
        self._check(self._lib.cc_mhd2d_compute_gravity(self._h, None, None))
        return None

    def compute_dt(self) -> float:
        dt = C.c_double()
        self._check(self._lib.cc_mhd2d_compute_dt(self._h, C.byref(dt)))
        return dt.value

    def rk2_step(self, g: GravField | None, dt: float):
        if g is None:
            self._check(self._lib.cc_mhd2d_rk2_step(self._h, None, None, float(dt)))
        else:
            self._check(self._lib.cc_mhd2d_rk2_step(self._h, _dp(g.gx), _dp(g.gy), float(dt)))

    def advance(self, nsteps: int, t: float | None = None) -> float:
        """nsteps of the main loop from time t (None: where the last advance,
        upload (t = 0) or checkpoint load left the clock); returns the time."""
        tt = C.c_double(getattr(self, "_t", 0.0) if t is None else t)
        self._check(self._lib.cc_mhd2d_advance(self._h, int(nsteps), C.byref(tt)))
        self._t = tt.value
        return tt.value

    def set_stage_kernel(self, kind: str, seg_rows: int = 0):
        """"tile" (the default) or "march" (FP32 only), seg_rows 0: chosen from
        the grid (cc_mhd2d_set_stage_kernel)."""
        k = {"tile": L.CC_STAGE_TILE, "march": L.CC_STAGE_MARCH}[kind]
        self._check(self._lib.cc_mhd2d_set_stage_kernel(self._h, k, int(seg_rows)))

    def set_stream(self, stream_ptr: int | None):
        """Issue work on a caller's cudaStream_t (e.g. torch's current stream)."""
        self._check(self._lib.cc_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def synchronize(self):
        self._check(self._lib.cc_synchronize(self._h))

    def set_profiling(self, on: bool):
        self._check(self._lib.cc_set_profiling(self._h, 1 if on else 0))

    def perf(self) -> dict:
        q = L.CcPerf()
        self._check(self._lib.cc_get_perf(self._h, C.byref(q)))
        return {f: getattr(q, f) for f, _ in L.CcPerf._fields_}

    def reset_perf(self):
        self._check(self._lib.cc_reset_perf(self._h))

    def diagnostics(self) -> dict:
        d = L.CcDiag()
        self._check(self._lib.cc_mhd2d_diagnostics(self._h, C.byref(d)))
        return {f: getattr(d, f) for f, _ in L.CcDiag._fields_}

    def derived(self) -> dict:
        """The reference main()'s snapshot fields (M2:1065-1106) of the resident
        state: {rho, P, Mach, u, v, vabs, Bx, By, Bz, divB}, each (Ny, Nx)."""
        n = self.p.Nx * self.p.Ny
        out = [np.empty(n) for _ in DERIVED_FIELDS]
        arr = (C.POINTER(C.c_double) * 10)(*[_dp(a) for a in out])
        self._check(self._lib.cc_mhd2d_derived(self._h, arr))
        return {k: a.reshape(self.p.Ny, self.p.Nx) for k, a in zip(DERIVED_FIELDS, out)}

    def save_checkpoint(self, path: str):
        """State, clock and parameters to one file (cc_mhd2d_checkpoint_save)."""
        self._check(self._lib.cc_mhd2d_checkpoint_save(self._h, str(path).encode()))

    def load_checkpoint(self, path: str):
        """Restore state and clock from a checkpoint of the same grid (cc_mhd2d_checkpoint_load)."""
        self._check(self._lib.cc_mhd2d_checkpoint_load(self._h, str(path).encode()))
        self._t = self.diagnostics()["t"]


# ---- drop-in functions with the reference's signatures ----

_cache: dict = {}


def _solver(p: Params) -> Mhd2dSolver:
    key = tuple(getattr(p, f.name) for f in fields(p))
    s = _cache.get(key)
    if s is None:
        if len(_cache) > 4:
            for v in _cache.values():
                v.close()
            _cache.clear()
        s = _cache[key] = Mhd2dSolver(p)
    return s


def compute_poisson_gravity_periodic(p: Params, rho: np.ndarray, dx: float, dy: float) -> GravField:
    """compute_poisson_gravity_periodic (M2:178-237) on the GPU."""
    s = _solver(p)
    U, B = empty_state(p)
    U.rho[:] = rho
    s.upload(U, B)
    return s.compute_gravity(to_host=True)


def compute_dt(p: Params, U: Ucc, B: Bfaces, dx: float, dy: float) -> float:
    """compute_dt (M2:579-598) on the GPU."""
    s = _solver(p)
    s.upload(U, B)
    return s.compute_dt()


def rk2_step(p: Params, U: Ucc, B: Bfaces, g: GravField, dx: float, dy: float, dt: float) -> None:
    """rk2_step (M2:838-869) on the GPU; U and B are updated in place."""
    s = _solver(p)
    s.upload(U, B)
    s.rk2_step(g, dt)
    s.download(U, B)


# ---- initial conditions (host side, libcc_b200's cc_ic_* functions) ----

def _ic_ptrs(U: Ucc, B: Bfaces):
    arr = (L._DP * 8)(*_state_ptrs(U, B))
    return arr


def ic_collapse(p: Params, core_amp: float = 9.0, core_width: float = 0.1, noise: float = 0.01, seed: int = 0,
                Bx0: float = 0.05, p0: float = 0.1, p_exponent: float = 5.0 / 3.0) -> tuple[Ucc, Bfaces]:
    U, B = empty_state(p)
    cp = p.to_c()
    r = L.lib().cc_ic_mhd2d_collapse(C.byref(cp), core_amp, core_width, noise, seed, Bx0, p0, p_exponent,
                                     _ic_ptrs(U, B))
    if r != 0:
        raise ValueError("cc_ic_mhd2d_collapse failed")
    return U, B


def ic_orszag_tang(p: Params, core_amp: float = 4.0, core_width: float = 0.1) -> tuple[Ucc, Bfaces]:
    U, B = empty_state(p)
    cp = p.to_c()
    if L.lib().cc_ic_mhd2d_orszag_tang(C.byref(cp), core_amp, core_width, _ic_ptrs(U, B)) != 0:
        raise ValueError("cc_ic_mhd2d_orszag_tang failed")
    return U, B


def ic_reference(p: Params, **knobs) -> tuple[Ucc, Bfaces]:
    U, B = empty_state(p)
    k = L.CcIcKnobs()
    L.lib().cc_mhd2d_ic_knobs_default(C.byref(k))
    for name, v in knobs.items():
        setattr(k, name, v)
    cp = p.to_c()
    if L.lib().cc_ic_mhd2d_reference(C.byref(cp), C.byref(k), _ic_ptrs(U, B)) != 0:
        raise ValueError("cc_ic_mhd2d_reference failed")
    return U, B
