"""Discrete adjoint of the 2D resistive-MHD step (include/cc_adjoint.h), and a
torch.autograd.Function over it.

`AdjointSolver` records a forward run of n steps of the reference's main-loop
body (mhd2d_resistive_hlld_ct_gravity.cpp:1111-1117; dt from the CFL rule,
recorded), keeps a checkpoint every k steps, and returns vector-Jacobian
products of the final state with respect to the initial state and eta.  dt
is a recorded constant of each step; gravity uses the direct Poisson solve.

`Mhd2dRollout.apply(rho0, eta, setup)` maps an initial density field and
eta to the density after `setup.nsteps` steps, differentiable in both.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, replace

import numpy as np

from . import _lib as L
from .mhd2d import Bfaces, CcError, Params, Ucc, _dp, empty_state


def _ptrs(U: Ucc, B: Bfaces):
    arrays = U.arrays() + [B.Bx_f, B.By_f]
    arr = (L._DP * 8)(*[_dp(a) for a in arrays])
    arr._keep = arrays
    return arr


class AdjointSolver:
    """One grid with a recorded, checkpointed forward run and its adjoint, in
    the precision of `p` ("fp64", or "fp32": FP32 forward and FP32 reverse
    kernels, eta's adjoint summed in FP64); states and adjoints cross the API
    as FP64 arrays.  Gravity: the direct Poisson solve, or "sor" (the
    single-grid red-black SOR with its recorded sweep counts, reversed sweep
    by sweep); "fft" is replaced by the direct solve."""

    def __init__(self, p: Params, checkpoint_every: int = 10, max_steps: int = 100):
        if p.gravity_on and p.poisson not in ("direct", "sor"):
            p = replace(p, poisson="direct")
        self.p = replace(p, compensated=False)
        self._lib = L.lib()
        self._cp = self.p.to_c()
        self._h = C.c_void_p()
        r = self._lib.cc_adjoint_create(C.byref(self._cp), int(checkpoint_every), int(max_steps), C.byref(self._h))
        if r != L.CC_OK:
            msg = self._lib.cc_last_error(self._h).decode() if self._h.value else "create failed"
            if self._h.value:
                self._lib.cc_destroy(self._h)
            self._h = C.c_void_p()
            raise CcError(r, msg)
        self.nsteps = 0

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

    def set_stream(self, stream: int):
        self._check(self._lib.cc_set_stream(self._h, C.c_void_p(stream)))

    def perf(self) -> dict:
        pf = L.CcPerf()
        self._check(self._lib.cc_get_perf(self._h, C.byref(pf)))
        return {f: getattr(pf, f) for f, _ in L.CcPerf._fields_}

    def upload(self, U: Ucc, B: Bfaces):
        self._check(self._lib.cc_adjoint_upload(self._h, _ptrs(U, B)))

    def forward(self, nsteps: int, t0: float = 0.0, replay: bool = False) -> float:
        t = C.c_double()
        self._check(self._lib.cc_adjoint_forward(self._h, int(nsteps), float(t0), 1 if replay else 0, C.byref(t)))
        self.nsteps = int(nsteps)
        return t.value

    def download(self) -> tuple[Ucc, Bfaces]:
        U, B = empty_state(self.p)
        self._check(self._lib.cc_adjoint_download(self._h, _ptrs(U, B)))
        return U, B

    def dts(self, n: int | None = None) -> np.ndarray:
        n = self.nsteps if n is None else n
        out = np.zeros(n)
        self._check(self._lib.cc_adjoint_get_dts(self._h, _dp(out), n))
        return out

    def set_dts(self, dts: np.ndarray):
        v = np.ascontiguousarray(dts, dtype=np.float64)
        self._check(self._lib.cc_adjoint_set_dts(self._h, _dp(v), len(v)))
        self.nsteps = len(v)

    def vjp(self, lamU: Ucc, lamB: Bfaces) -> tuple[Ucc, Bfaces, float]:
        """Adjoint of the initial state and of eta for the recorded run."""
        U0, B0 = empty_state(self.p)
        eta = C.c_double()
        self._check(self._lib.cc_adjoint_vjp(self._h, _ptrs(lamU, lamB), _ptrs(U0, B0), C.byref(eta)))
        return U0, B0, eta.value


def density_loss_adjoint(p: Params, rho_T: np.ndarray, target: np.ndarray) -> tuple[float, Ucc, Bfaces]:
    """0.5 sum (rho_T - target)^2 and its adjoint on the final state."""
    d = rho_T - target
    lamU, lamB = empty_state(p)
    lamU.rho[:] = d
    return 0.5 * float(d @ d), lamU, lamB


@dataclass
class RolloutSetup:
    """Fixed part of a differentiable rollout: parameters (eta is the
    differentiable argument), the non-density initial fields, the step count
    and the checkpoint interval."""
    params: Params
    U0: Ucc
    B0: Bfaces
    nsteps: int
    checkpoint_every: int = 10


try:
    import torch

    class Mhd2dRollout(torch.autograd.Function):
        """rho_T = F(rho0, eta): nsteps of the 2D MHD step from the initial
        state of `setup` with its density replaced by rho0 (flat, Nx*Ny,
        float64).  backward returns the discrete-adjoint gradients with
        respect to rho0 and eta (dt recorded in the forward run)."""

        @staticmethod
        def forward(ctx, rho0, eta, setup: RolloutSetup):
            p = replace(setup.params, eta=float(eta))
            s = AdjointSolver(p, setup.checkpoint_every, max(setup.nsteps, 1))
            U = setup.U0.copy()
            U.rho[:] = rho0.detach().cpu().numpy().astype(np.float64)
            s.upload(U, setup.B0)
            s.forward(setup.nsteps)
            UT, _ = s.download()
            ctx.solver = s
            return torch.from_numpy(UT.rho.copy())

        @staticmethod
        def backward(ctx, grad_rho):
            s: AdjointSolver = ctx.solver
            lamU, lamB = empty_state(s.p)
            lamU.rho[:] = grad_rho.detach().cpu().numpy().astype(np.float64)
            l0, _, leta = s.vjp(lamU, lamB)
            s.close()
            return torch.from_numpy(l0.rho.copy()), torch.tensor(leta, dtype=torch.float64), None
except ImportError:   # torch is optional for the C-ABI wrapper above
    pass
