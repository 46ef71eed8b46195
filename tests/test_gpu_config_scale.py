"""GPU parity at the scale of the benchmark workloads, against the CPU oracle
(the restatement of the reference step, pinned bit for bit to the reference
compiled in place by the test_oracle_pin_* tests).

* FFT-gravity workload (periodic [-1,1]^2, Orszag-Tang fields + Gaussian core
  of amplitude 4 and width 0.1, gamma 5/3, G 1, eta 1e-3, CFL 0.4):
  - 256^2, 20 main-loop steps, FP64: relative L-inf <= 1e-12 per field;
  - 1024^2 (the smaller grid of the precision ladder), FP64: <= 1e-12 after
    ORACLE_STEPS_1024 steps, as many as the CPU oracle runs in about a minute;
  - 1024^2 FP32 to the same final time: per-field L1 and L-inf against the
    FP64 oracle, printed, L1 <= 1e-5 (the FP32 target).
* Outflow collapse workload (256^2, core amplitude 9, width 0.1, 1% noise
  seed 0, p = 0.1 rho^(5/3), Bx 0.05, eta 1e-3, G 1, CFL 0.4, red-black SOR
  omega 1.9 with the reference's fixed 600 sweeps): 10 steps, FP64, <= 1e-12
  against the oracle's red-black SOR.
* 3D workload physics (ideal gas gamma 5/3, eta 5e-4, random-phase v and A,
  seed 1) at 64^3: 3 steps, FP64, <= 1e-12.

FP64 tolerance: the GPU rounds like the reference except in the order of the
density / potential mean sums (a fixed tree instead of a running sum)."""
import numpy as np
import pytest

import oracle_lib as O
from core_collapse_b200.mhd2d import Mhd2dSolver, Params, ic_collapse, ic_orszag_tang
from core_collapse_b200.mhd3d import Mhd3dSolver, Params3, ic_turbulence3d

pytestmark = pytest.mark.gpu

TOL = 1e-12
FP32_L1 = 1e-5
ORACLE_STEPS_1024 = 24
FIELDS = ["rho", "mx", "my", "mz", "E", "Bz", "Bx_f", "By_f"]


def _fft_params(n: int, precision: str) -> Params:
    return Params(Nx=n, Ny=n, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=True, periodic_y=True, gamma=5.0 / 3.0,
                  G=1.0, eta=1e-3, cfl=0.4, gravity_on=True, poisson="fft", precision=precision, t_end=1e30)


def _worst(got, want):
    return max((O.rel_linf(a, b), FIELDS[k]) for k, (a, b) in enumerate(zip(got, want)))


def _run_gpu(p, U, B, nsteps):
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        t = s.advance(nsteps, 0.0)
        U2, B2 = s.download()
        d = s.diagnostics()
    return O.state_list(U2, B2), t, d


def test_fft_workload_256_fp64_20_steps():
    p = _fft_params(256, "fp64")
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.1)
    want, t_want = O.m2_main_loop_oracle(p.to_c(), O.state_list(U, B), 20, mode=2)
    got, t, d = _run_gpu(p, U, B, 20)
    assert d["steps"] == 20
    assert abs(t - t_want) <= 1e-12 * t_want
    err, name = _worst(got, want)
    print(f"256^2 FFT workload, 20 steps FP64: max rel L-inf {err:.2e} ({name})")
    assert err <= TOL, f"{name}: {err:.3e}"


@pytest.fixture(scope="module")
def oracle_1024():
    p = _fft_params(1024, "fp64")
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.1)
    want, t_want = O.m2_main_loop_oracle(p.to_c(), O.state_list(U, B), ORACLE_STEPS_1024, mode=2)
    return U, B, want, t_want


def test_fft_workload_1024_fp64(oracle_1024):
    U, B, want, t_want = oracle_1024
    got, t, _ = _run_gpu(_fft_params(1024, "fp64"), U, B, ORACLE_STEPS_1024)
    assert abs(t - t_want) <= 1e-12 * t_want
    err, name = _worst(got, want)
    print(f"1024^2 FFT workload, {ORACLE_STEPS_1024} steps FP64: max rel L-inf {err:.2e} ({name})")
    assert err <= TOL, f"{name}: {err:.3e}"


def test_fft_workload_1024_fp32_error(oracle_1024):
    """FP32 bulk path to the oracle's final time (its own CFL steps, the last
    one clamped): per-field relative L1 and L-inf against the FP64 oracle."""
    U, B, want, t_want = oracle_1024
    p = _fft_params(1024, "fp32")
    p.t_end = t_want
    got, t, d = _run_gpu(p, U, B, ORACLE_STEPS_1024 + 8)
    assert abs(t - t_want) <= 1e-12 * t_want
    l1 = {}
    linf = {}
    for k, (a, b) in enumerate(zip(got, want)):
        den = float(np.sum(np.abs(b)))
        l1[FIELDS[k]] = float(np.sum(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a)))
        linf[FIELDS[k]] = O.rel_linf(a, b)
    print(f"1024^2 FFT workload, FP32 vs FP64 oracle at t={t:.6e} ({d['steps']} steps):")
    for k in FIELDS:
        print(f"  {k:5s} L1 {l1[k]:.2e}  L-inf {linf[k]:.2e}")
    assert max(l1.values()) <= FP32_L1
    assert max(linf.values()) <= 1e-2


def test_collapse_sor_256_fp64_10_steps():
    p = Params(Nx=256, Ny=256, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=False, periodic_y=False,
               gamma=5.0 / 3.0, G=1.0, eta=1e-3, cfl=0.4, gravity_on=True, poisson="sor", sor_iters=600,
               sor_omega=1.9, precision="fp64", t_end=1e30)
    U, B = ic_collapse(p, core_amp=9.0, core_width=0.1, noise=0.01, seed=0, Bx0=0.05)
    want, t_want = O.m2_main_loop_oracle(p.to_c(), O.state_list(U, B), 10, mode=1)
    got, t, d = _run_gpu(p, U, B, 10)
    assert d["steps"] == 10
    assert abs(t - t_want) <= 1e-12 * t_want
    err, name = _worst(got, want)
    print(f"256^2 collapse workload, SOR 600 sweeps, 10 steps FP64: max rel L-inf {err:.2e} ({name})")
    assert err <= TOL, f"{name}: {err:.3e}"


def test_turbulence3d_64_fp64_3_steps():
    n = 64
    p = Params3.ideal_gas(Nx=n, Ny=n, Nz=n, eta=5e-4, cfl=0.4, precision="fp64", t_end=1e30)
    s0 = ic_turbulence3d(Params3.ideal_gas(Nx=n, Ny=n, Nz=n), seed=1)
    want, t_want = O.m3_main_loop_oracle(p.to_c(), [a.copy() for a in s0.arrays()], 3)
    with Mhd3dSolver(p) as g:
        g.upload(s0)
        t = g.advance(3, 0.0)
        got = g.download().arrays()
    assert abs(t - t_want) <= 1e-12 * t_want
    names = ["rho", "mx", "my", "mz", "E", "Bx_f", "By_f", "Bz_f"]
    err, k = max((O.rel_linf(a, b), k) for k, (a, b) in enumerate(zip(got, want)))
    print(f"64^3 turbulence workload, 3 steps FP64: max rel L-inf {err:.2e} ({names[k]})")
    assert err <= TOL, f"{names[k]}: {err:.3e}"
