"""The column-march FP32 stage kernel (CC_STAGE_MARCH, mhd2d_march.cuh)
against the tile stage kernel (CC_STAGE_TILE) on the same inputs: same
expressions, different work distribution (carried rows instead of a
recomputed halo), so the two agree to FP32 contraction-level differences.
Covered: every seeded 2D case (periodic, outflow and mixed boundaries,
gravity arrays / potential, resistive and ideal, the HLL fallback, floors),
grids that are not multiples of the strip width, segments that are not
multiples of the march step, one-row segments, and the compensated state."""
import numpy as np
import pytest

import oracle_lib as O
from cases_mhd2d import CASES, make_case
from core_collapse_b200.mhd2d import Mhd2dSolver, Params, ic_collapse, ic_orszag_tang

pytestmark = pytest.mark.gpu

TOL = 2e-5   # relative L-inf per field after a few steps, FP32


def _run(p, U, B, nsteps, kind, seg=0):
    with Mhd2dSolver(p) as s:
        s.set_stage_kernel(kind, seg)
        s.upload(U, B)
        t = s.advance(nsteps, 0.0)
        return O.state_list(*s.download()), t


def _compare(a_list, b_list, what):
    worst = max(O.rel_linf(a, b) for a, b in zip(a_list, b_list))
    same = all(np.array_equal(a, b) for a, b in zip(a_list, b_list))
    print(f"{what}: march vs tile max rel L-inf {worst:.2e}{' (bit-identical)' if same else ''}")
    assert worst <= TOL, f"{what}: {worst:.3e}"


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("seg", [0, 128, 5, 1])
def test_march_matches_tile_cases(name, seg):
    p, U, B = make_case(name, precision="fp32")
    p.t_end = 10.0
    a, ta = _run(p, U, B, 4, "march", seg)
    b, tb = _run(p, U, B, 4, "tile")
    assert abs(ta - tb) <= 1e-6 * tb
    _compare(a, b, f"{name} seg {seg}")


@pytest.mark.parametrize("compensated", [False, True])
def test_march_matches_tile_fft_ragged(compensated):
    # 128 columns = 4 strips, 64 rows in segments of 20 (steps of 8, 8, 4)
    p = Params(Nx=128, Ny=64, x0=-1, x1=1, y0=-1, y1=1, eta=1e-3, G=1.0, gravity_on=True, poisson="fft",
               precision="fp32", compensated=compensated, cfl=0.4, t_end=10.0)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.2)
    a, _ = _run(p, U, B, 6, "march", 20)
    b, _ = _run(p, U, B, 6, "tile")
    _compare(a, b, f"FFT 128x64 compensated={compensated}")


def test_march_matches_tile_outflow_odd_grid():
    p = Params(Nx=100, Ny=70, x0=-1, x1=1, y0=-1, y1=1, periodic_x=False, periodic_y=False, eta=2e-3, G=1.0,
               gravity_on=True, poisson="sor", sor_iters=50, sor_omega=1.9, precision="fp32", cfl=0.4, t_end=10.0)
    U, B = ic_collapse(p, core_amp=9.0, core_width=0.2, noise=0.01, seed=3, Bx0=0.05)
    a, _ = _run(p, U, B, 5, "march", 33)
    b, _ = _run(p, U, B, 5, "tile")
    _compare(a, b, "outflow 100x70 SOR")


def test_march_rejected_for_fp64():
    from core_collapse_b200.mhd2d import CcError
    p = Params(Nx=32, Ny=32, precision="fp64")
    with Mhd2dSolver(p) as s, pytest.raises(CcError):
        s.set_stage_kernel("march", 64)
