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


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "state arrays must be contiguous float64"
    return a.ctypes.data_as(L._DP)


# output order of the reference's snapshot store (M3:1309-1319)
DERIVED3_FIELDS = ("rho", "P", "Mach", "u", "v", "w", "vabs", "Bx", "By", "Bz", "divB")


def ic_reference3(p: Params3, **knobs) -> State3:
    """The 3D reference main()'s core-collapse IC (M3:1159-1272); knobs
    override cc_mhd3d_ic_knobs_default (rho_bg, rho_core, r_core, r_edge, P0,
    vin, rot_omega, B0x, B0z, Bshear)."""
    s = empty_state3(p)
    k = L.CcIc3Knobs()
    L.lib().cc_mhd3d_ic_knobs_default(C.byref(k))
    for name, v in knobs.items():
        setattr(k, name, float(v))
    arr = (C.POINTER(C.c_double) * 8)(*[_dp(a) for a in s.arrays()])
    cp = p.to_c()
    if L.lib().cc_ic_mhd3d_reference(C.byref(cp), C.byref(k), arr) != 0:
        raise ValueError("cc_ic_mhd3d_reference rejected its arguments")
    return s


class Mhd3dSolver:
    """A device-resident 3D MHD instance (one libcc_b200 handle)."""

    def __init__(self, p: Params3):
        from .mhd2d import CcError
        self._Err = CcError
        self.p = p
        self._lib = L.lib()
        self._cp = p.to_c()
        self._h = C.c_void_p()
        r = self._lib.cc_mhd3d_create(C.byref(self._cp), C.byref(self._h))
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

    def upload(self, s: State3):
        self._check(self._lib.cc_mhd3d_upload(self._h, *[_dp(a) for a in s.arrays()]))
        self._t = 0.0

    def download(self, s: State3 | None = None) -> State3:
        if s is None:
            s = empty_state3(self.p)
        self._check(self._lib.cc_mhd3d_download(self._h, *[_dp(a) for a in s.arrays()]))
        return s

    def compute_dt(self) -> float:
        dt = C.c_double()
        self._check(self._lib.cc_mhd3d_compute_dt(self._h, C.byref(dt)))
        return dt.value

    def rk2_step(self, dt: float):
        self._check(self._lib.cc_mhd3d_rk2_step(self._h, float(dt)))

    def advance(self, nsteps: int, t: float | None = None) -> float:
        """nsteps of the main loop from time t (None: where the last advance or
        upload (t = 0) left the clock); returns the time."""
        tt = C.c_double(getattr(self, "_t", 0.0) if t is None else t)
        self._check(self._lib.cc_mhd3d_advance(self._h, int(nsteps), C.byref(tt)))
        self._t = tt.value
        return tt.value

    def set_stream(self, stream_ptr: int | None):
        self._check(self._lib.cc_set_stream(self._h, C.c_void_p(stream_ptr) if stream_ptr else None))

    def set_profiling(self, on: bool):
        self._check(self._lib.cc_set_profiling(self._h, 1 if on else 0))

    def perf(self) -> dict:
        q = L.CcPerf()
        self._check(self._lib.cc_get_perf(self._h, C.byref(q)))
        return {f: getattr(q, f) for f, _ in L.CcPerf._fields_}

    def reset_perf(self):
        self._check(self._lib.cc_reset_perf(self._h))

    def save_checkpoint(self, path: str):
        """State, clock and parameters to one file (cc_mhd3d_checkpoint_save)."""
        self._check(self._lib.cc_mhd3d_checkpoint_save(self._h, str(path).encode()))

    def load_checkpoint(self, path: str):
        """Restore state and clock from a checkpoint of the same grid (cc_mhd3d_checkpoint_load)."""
        self._check(self._lib.cc_mhd3d_checkpoint_load(self._h, str(path).encode()))
        self._t = self.diagnostics()["t"]

    def diagnostics(self) -> dict:
        d = L.CcDiag()
        self._check(self._lib.cc_mhd3d_diagnostics(self._h, C.byref(d)))
        return {f: getattr(d, f) for f, _ in L.CcDiag._fields_}

    def derived(self) -> dict:
        """The reference main()'s snapshot fields (M3:1293-1321), each (Nz, Ny, Nx)."""
        n = self.p.Nx * self.p.Ny * self.p.Nz
        out = [np.empty(n) for _ in DERIVED3_FIELDS]
        arr = (C.POINTER(C.c_double) * 11)(*[_dp(a) for a in out])
        self._check(self._lib.cc_mhd3d_derived(self._h, arr))
        return {k: a.reshape(self.p.Nz, self.p.Ny, self.p.Nx) for k, a in zip(DERIVED3_FIELDS, out)}


# ---- drop-in functions with the reference's signatures (M3:626, 1034) ----

def compute_dt(p: Params3, s: State3, dx: float, dy: float, dz: float) -> float:
    with Mhd3dSolver(p) as g:
        g.upload(s)
        return g.compute_dt()


def rk2_step(p: Params3, s: State3, dx: float, dy: float, dz: float, dt: float) -> None:
    """rk2_step on the GPU; the state arrays are updated in place."""
    with Mhd3dSolver(p) as g:
        g.upload(s)
        g.rk2_step(dt)
        g.download(s)


# ---- initial conditions (host side) ----

def _random_phase_field(shape, offset, modes, phases, amp=1.0):
    """Re sum_n amp e^{i phase_n} e^{2 pi i n.(j + offset)/N} at grid indices j of
    `shape` = (Nz, Ny, Nx), for integer mode vectors `modes` (m, 3) as (nx, ny, nz)."""
    nz, ny, nx = shape
    F = np.zeros(shape, dtype=np.complex128)
    shift = np.exp(2j * np.pi * (modes[:, 0] * offset[0] / nx + modes[:, 1] * offset[1] / ny +
                                 modes[:, 2] * offset[2] / nz))
    np.add.at(F, (modes[:, 2] % nz, modes[:, 1] % ny, modes[:, 0] % nx), amp * np.exp(1j * phases) * shift)
    return np.real(np.fft.ifftn(F)) * (nx * ny * nz)


def ic_turbulence3d(p: Params3, seed: int = 1, v_rms: float = 0.5, b_rms: float = 0.3, kmin: float = 1.0,
                    kmax: float = 4.0, rho0: float = 1.0, gamma: float = 5.0 / 3.0) -> State3:
    """Uniform density rho0 and pressure 1/gamma; velocity and edge vector
    potential A are random-phase Fourier fields over the integer mode vectors
    with kmin <= |n| <= kmax (one numpy Generator(seed) draws every phase);
    v is scaled to rms v_rms over cells, B = curl A on faces (div B = 0 to
    roundoff) scaled so the cell-centred |B| has rms b_rms.  Periodic box."""
    nx, ny, nz = p.Nx, p.Ny, p.Nz
    rng = np.random.default_rng(seed)
    r = int(np.ceil(kmax))
    g = np.arange(-r, r + 1)
    M = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    kk = np.sqrt((M ** 2).sum(1))
    modes = M[(kk >= kmin) & (kk <= kmax)]
    ph = rng.uniform(0.0, 2.0 * np.pi, size=(6, len(modes)))
    shape = (nz, ny, nx)
    v = [_random_phase_field(shape, (0.5, 0.5, 0.5), modes, ph[c]) for c in range(3)]
    vs = v_rms / np.sqrt(np.mean(v[0] ** 2 + v[1] ** 2 + v[2] ** 2))
    u, vv, w = (a.ravel() * vs for a in v)
    Ax = _random_phase_field(shape, (0.5, 0.0, 0.0), modes, ph[3])   # x-edges (i+1/2, j, k)
    Ay = _random_phase_field(shape, (0.0, 0.5, 0.0), modes, ph[4])   # y-edges (i, j+1/2, k)
    Az = _random_phase_field(shape, (0.0, 0.0, 0.5), modes, ph[5])   # z-edges (i, j, k+1/2)
    dx, dy, dz = p.dx, p.dy, p.dz
    roll = lambda a, ax: np.roll(a, -1, axis=ax)   # value at index + 1 (periodic)
    # cell-indexed faces, then the face at index N repeats face 0
    bx = (roll(Az, 1) - Az) / dy - (roll(Ay, 0) - Ay) / dz
    by = (roll(Ax, 0) - Ax) / dz - (roll(Az, 2) - Az) / dx
    bz = (roll(Ay, 2) - Ay) / dx - (roll(Ax, 1) - Ax) / dy
    bxc, byc, bzc = 0.5 * (bx + roll(bx, 2)), 0.5 * (by + roll(by, 1)), 0.5 * (bz + roll(bz, 0))
    bs = b_rms / np.sqrt(np.mean(bxc ** 2 + byc ** 2 + bzc ** 2))
    bx, by, bz, bxc, byc, bzc = (a * bs for a in (bx, by, bz, bxc, byc, bzc))
    Bx_f = np.concatenate([bx, bx[:, :, :1]], axis=2)
    By_f = np.concatenate([by, by[:, :1, :]], axis=1)
    Bz_f = np.concatenate([bz, bz[:1, :, :]], axis=0)
    n = nx * ny * nz
    rho = np.full(n, rho0)
    P = 1.0 / gamma
    E = 0.5 * rho * (u * u + vv * vv + w * w) + 0.5 * (bxc.ravel() ** 2 + byc.ravel() ** 2 + bzc.ravel() ** 2) + \
        P / (gamma - 1.0)
    return State3(rho, rho * u, rho * vv, rho * w, E, Bx_f.ravel().copy(), By_f.ravel().copy(), Bz_f.ravel().copy())
