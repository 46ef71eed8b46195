"""Batched ensemble of independent 2D resistive-MHD instances on one GPU
(include/cc_batch.h).

Each instance is a `Params` of the single-grid solver (its own grid, domain,
boundaries, physics constants, t_end); the ensemble advances all of them with
one persistent stage kernel per RK stage over a tile work-list and a per-
instance dt.  Instances with gravity use the direct Poisson solve
(`Params.poisson = "direct"`): the exact solution of the discrete problem the
reference's SOR (mhd2d_resistive_hlld_ct_gravity.cpp:207-223) iterates
towards.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import replace

import numpy as np

from . import _lib as L
from .mhd2d import Bfaces, CcError, Params, Ucc, _dp, empty_state, ic_collapse


def _ptr_array(arrays) -> C.Array:
    arr = (L._DP * len(arrays))(*[_dp(a) for a in arrays])
    arr._keep = arrays
    return arr


class BatchSolver:
    """n device-resident instances advanced together (one libcc_b200 handle)."""

    def __init__(self, params: list[Params]):
        if not params:
            raise ValueError("empty ensemble")
        self.params = list(params)
        self.n = len(self.params)
        self._lib = L.lib()
        self._cp = (L.CcMhd2dParams * self.n)(*[p.to_c() for p in self.params])
        self._h = C.c_void_p()
        r = self._lib.cc_batch_create(self._cp, self.n, C.byref(self._h))
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
    def handle(self) -> int:
        return self._h.value

    def set_stream(self, stream: int):
        self._check(self._lib.cc_set_stream(self._h, C.c_void_p(stream)))

    def upload(self, i: int, U: Ucc, B: Bfaces):
        self._check(self._lib.cc_batch_upload(self._h, i, _ptr_array(U.arrays() + [B.Bx_f, B.By_f])))

    def download(self, i: int) -> tuple[Ucc, Bfaces]:
        U, B = empty_state(self.params[i])
        self._check(self._lib.cc_batch_download(self._h, i, _ptr_array(U.arrays() + [B.Bx_f, B.By_f])))
        return U, B

    def compute_dt(self) -> np.ndarray:
        dt = np.zeros(self.n)
        self._check(self._lib.cc_batch_compute_dt(self._h, _dp(dt)))
        return dt

    def advance(self, nsteps: int, t: np.ndarray | None = None) -> np.ndarray:
        """nsteps of every instance's main-loop body; returns the instances' times."""
        tt = np.zeros(self.n) if t is None else np.ascontiguousarray(t, dtype=np.float64).copy()
        ptr = _dp(tt) if t is not None else None
        self._check(self._lib.cc_batch_advance(self._h, int(nsteps), ptr))
        if t is None:
            self._check(self._lib.cc_batch_times(self._h, _dp(tt)))
        return tt

    def times(self) -> np.ndarray:
        """Every instance's simulated time (one device-to-host copy)."""
        tt = np.zeros(self.n)
        self._check(self._lib.cc_batch_times(self._h, _dp(tt)))
        return tt

    def diagnostics(self, i: int) -> dict:
        d = L.CcDiag()
        self._check(self._lib.cc_batch_diagnostics(self._h, i, C.byref(d)))
        return {f: getattr(d, f) for f, _ in L.CcDiag._fields_}

    def autotune(self, reps: int = 5) -> tuple[int, float]:
        shape, ms = C.c_int(), C.c_double()
        self._check(self._lib.cc_batch_autotune(self._h, reps, C.byref(shape), C.byref(ms)))
        return shape.value, ms.value

    def set_shape(self, shape: int):
        self._check(self._lib.cc_batch_set_shape(self._h, shape))

    def info(self) -> dict:
        o = L.CcBatchInfo()
        self._check(self._lib.cc_batch_get_info(self._h, C.byref(o)))
        return {f: getattr(o, f) for f, _ in L.CcBatchInfo._fields_}

    def set_profiling(self, on: bool):
        """Bracket stage launches with CUDA events (time loops then run without graphs)."""
        self._check(self._lib.cc_set_profiling(self._h, 1 if on else 0))

    def reset_perf(self):
        self._check(self._lib.cc_reset_perf(self._h))

    def perf(self) -> dict:
        pf = L.CcPerf()
        self._check(self._lib.cc_get_perf(self._h, C.byref(pf)))
        return {f: getattr(pf, f) for f, _ in L.CcPerf._fields_}


def collapse_ensemble(n: int, seed: int = 2, sides=(64, 96, 128, 192, 256), precision: str = "fp32",
                      t_end: float = 1e30) -> tuple[list[Params], list[tuple[Ucc, Bfaces]]]:
    """An ensemble of 2D collapse instances: the 256^2 collapse physics on
    [-1,1]^2 with outflow boundaries (gamma 5/3, G 1, CFL 0.4), side drawn
    uniformly from `sides`, core amplitude U(2,20), core width U(0.05,0.2),
    Bx U(0,0.2), eta log-uniform in [1e-4, 1e-2]; density noise 1% from
    std::mt19937(instance index); p = 0.1 rho^(5/3)."""
    rng = np.random.default_rng(seed)
    base = Params(x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=False, periodic_y=False, gamma=5.0 / 3.0, G=1.0,
                  cfl=0.4, gravity_on=True, poisson="direct", precision=precision, t_end=t_end)
    params, states = [], []
    for i in range(n):
        side = int(rng.choice(sides))
        amp = float(rng.uniform(2.0, 20.0))
        width = float(rng.uniform(0.05, 0.2))
        bx = float(rng.uniform(0.0, 0.2))
        eta = float(10.0 ** rng.uniform(-4.0, -2.0))
        p = replace(base, Nx=side, Ny=side, eta=eta)
        U, B = ic_collapse(p, core_amp=amp, core_width=width, noise=0.01, seed=i, Bx0=bx, p0=0.1,
                           p_exponent=5.0 / 3.0)
        params.append(p)
        states.append((U, B))
    return params, states


def partition_by_cells(params: list[Params], world: int) -> list[list[int]]:
    """Split instance indices over `world` GPUs, balancing cells: largest
    instance first onto the least-loaded GPU (ties to the lower rank), each
    GPU's list kept in instance order.  The ensemble needs no collective
    inside a step; ranks only gather results at the end."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(params)), key=lambda i: (-params[i].Nx * params[i].Ny, i))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += params[i].Nx * params[i].Ny
    return [sorted(pl) for pl in parts]


def gather_by_instance(local: dict[int, object], world: int) -> dict[int, object]:
    """All-gather per-instance results {instance: value} from every rank
    (torch.distributed, any backend) into one dict on every rank."""
    if world == 1:
        return dict(local)
    import torch.distributed as dist
    out: list = [None] * world
    dist.all_gather_object(out, local)
    merged: dict[int, object] = {}
    for d in out:
        merged.update(d)
    return merged
