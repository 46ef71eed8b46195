"""cc_mhd2d_gravity_fft_noalloc: the spectral gravity solve for callers that
cannot allocate device memory (their GPU memory is owned by another memory
manager, or their loop must not pay cudaMalloc's implicit synchronisation).
Its scratch is a fixed array inside the library; the test allocates the input
and output device buffers itself (with torch) and calls the entry point
through the C ABI twice in a row, on different densities, checking each result
against cc_mhd2d_compute_gravity (FFT, FP64) on the same density within the
FP64 parity tolerance.

This file is collected last on purpose (test_zz_*): it also has to pass when
run alone in a fresh process."""
import ctypes as C

import numpy as np
import pytest

from core_collapse_b200 import _lib as L
from core_collapse_b200.mhd2d import Mhd2dSolver, Params, ic_orszag_tang

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative L-inf, the FP64 parity tolerance of the GPU tests


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _noalloc(p: Params, rho_dev, gx_dev, gy_dev, stream) -> int:
    cp = p.to_c()
    return L.lib().cc_mhd2d_gravity_fft_noalloc(C.byref(cp), C.c_void_p(rho_dev.data_ptr()),
                                                C.c_void_p(gx_dev.data_ptr()), C.c_void_p(gy_dev.data_ptr()),
                                                C.c_void_p(stream.cuda_stream))


def test_noalloc_gravity_matches_compute_gravity_twice():
    import torch
    p = Params(Nx=256, Ny=128, x0=-1, x1=1, y0=-1, y1=1, G=1.0, gravity_on=True, poisson="fft", precision="fp64")
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.2)
    rng = np.random.default_rng(5)
    densities = [U.rho.copy(), U.rho * (1.0 + 0.2 * rng.random(U.rho.size))]
    stream = torch.cuda.Stream()
    for rho in densities:
        U.rho[:] = rho
        with Mhd2dSolver(p) as s:
            s.upload(U, B)
            want = s.compute_gravity()
        rho_dev = torch.from_numpy(rho).to("cuda")
        gx_dev = torch.full_like(rho_dev, float("nan"))
        gy_dev = torch.full_like(rho_dev, float("nan"))
        torch.cuda.synchronize()
        assert _noalloc(p, rho_dev, gx_dev, gy_dev, stream) == L.CC_OK
        stream.synchronize()
        gx, gy = gx_dev.cpu().numpy(), gy_dev.cpu().numpy()
        assert np.all(np.isfinite(gx)) and np.all(np.isfinite(gy))
        assert _rel(gx, want.gx) <= TOL and _rel(gy, want.gy) <= TOL


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    p = Params(Nx=1024, Ny=1024, x0=-1, x1=1, y0=-1, y1=1, poisson="fft", precision="fp64")
    assert p.Nx * p.Ny > L.CC_NOALLOC_MAX_CELLS
    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    assert _noalloc(p, t, t, t, torch.cuda.current_stream()) == L.CC_ERR_TOO_LARGE


def test_noalloc_rejects_other_solvers_and_precisions():
    import torch
    t = torch.zeros(64 * 64, dtype=torch.float64, device="cuda")
    for kw in ({"poisson": "sor"}, {"poisson": "direct"}, {"poisson": "fft", "precision": "fp32"},
               {"poisson": "fft", "periodic_x": False}):
        p = Params(**{"Nx": 64, "Ny": 64, "x0": -1, "x1": 1, "y0": -1, "y1": 1, "precision": "fp64", **kw})
        assert _noalloc(p, t, t, t, torch.cuda.current_stream()) == L.CC_ERR_UNSUPPORTED, kw
