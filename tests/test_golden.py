"""Pin the CPU oracle to golden fixtures written by the compiled reference.

tests/golden/*.npz hold seeded inputs and the reference's own outputs
(tests/golden/make_golden.py): compute_dt, one advance_stage, one rk2_step
and a 3-step main-loop body of each solver, the reference's SOR gravity, its
random-blob IC and its radix-2 FFT.  The oracle must reproduce every value
bit for bit.  These tests need neither the reference tree nor a GPU."""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O
from core_collapse_b200.euler2d import ParamsEH
from core_collapse_b200.mhd2d import Params
from core_collapse_b200.mhd3d import Params3

GOLDEN = Path(__file__).resolve().parent / "golden"
_KIND = {"mhd2d": Params, "mhd3d": Params3, "euler2d": ParamsEH}


def _files(prefix):
    return sorted(p.stem for p in GOLDEN.glob(f"{prefix}_*.npz"))


def _load(stem):
    z = np.load(GOLDEN / f"{stem}.npz")
    meta = json.loads(str(z["params"]))
    p = _KIND[meta["kind"]](**meta["fields"])
    return p, z


def _state(z, prefix):
    keys = sorted((k for k in z.files if k.startswith(prefix) and k[len(prefix):].isdigit()),
                  key=lambda k: int(k[len(prefix):]))
    return [z[k].copy() for k in keys]


def _same(got, want):
    assert len(got) == len(want)
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"field {k}: max |d| = {np.max(np.abs(a - b))}"


def test_fixtures_present():
    assert len(_files("mhd2d")) >= 5 and len(_files("mhd3d")) >= 4 and len(_files("euler2d")) >= 4
    assert (GOLDEN / "fft.npz").exists()


@pytest.mark.parametrize("stem", _files("mhd2d"))
def test_mhd2d_golden(stem):
    p, z = _load(stem)
    cp = p.to_c()
    S = _state(z, "in")
    assert O.oracle().or_mhd2d_compute_dt(C.byref(cp), O.pp(S)) == float(z["dt"])
    if p.gravity_on:
        gx, gy, it, _ = O.m2_gravity_oracle(cp, S[0], mode=0)
        assert it == p.sor_iters
        _same([gx, gy], [z["gx"], z["gy"]])
    gx, gy, dt = z["gx"].copy(), z["gy"].copy(), float(z["dt"])
    _same(O.m2_stage_oracle(cp, S, gx, gy, dt), _state(z, "stage"))
    _same(O.m2_rk2_oracle(cp, S, gx, gy, dt, mode=0), _state(z, "step"))
    cp.t_end = 10.0
    loop, t = O.m2_main_loop_oracle(cp, S, 3, mode=0)
    assert t == float(z["loop_t"])
    _same(loop, _state(z, "loop"))
    assert O.oracle().or_mhd2d_divB_max(C.byref(cp), O.pp(loop)) == float(z["loop_divb"])


@pytest.mark.parametrize("stem", _files("mhd3d"))
def test_mhd3d_golden(stem):
    p, z = _load(stem)
    cp = p.to_c()
    S = _state(z, "in")
    dt = float(z["dt"])
    assert O.oracle().or_mhd3d_compute_dt(C.byref(cp), O.pp(S)) == dt
    stage = O.copy_state(S)
    O.oracle().or_mhd3d_advance_stage(C.byref(cp), O.pp(S), O.pp(stage), dt)
    _same(stage, _state(z, "stage"))
    _same(O.m3_rk2_oracle(cp, S, dt), _state(z, "step"))
    cp.t_end = 10.0
    loop, t = O.m3_main_loop_oracle(cp, S, 3)
    assert t == float(z["loop_t"])
    _same(loop, _state(z, "loop"))
    assert O.oracle().or_mhd3d_divB_max(C.byref(cp), O.pp(loop)) == float(z["loop_divb"])


@pytest.mark.parametrize("stem", [s for s in _files("euler2d") if s != "euler2d_random_blob"])
def test_euler2d_golden(stem):
    p, z = _load(stem)
    cp = p.to_c()
    S = _state(z, "in")
    dt = float(z["dt"])
    assert O.oracle().or_euler2d_compute_dt(C.byref(cp), O.pp(S)) == dt
    rhs = [np.zeros_like(a) for a in S]
    O.oracle().or_euler2d_rhs(C.byref(cp), O.pp(S), O.pp(rhs), 0)
    _same(rhs, _state(z, "rhs"))
    step = O.copy_state(S)
    O.oracle().or_euler2d_rk2_step(C.byref(cp), O.pp(step), dt, 0)
    _same(step, _state(z, "step"))


def test_euler2d_random_blob_golden():
    """The reference main(): its IC (restated twice: oracle loop input and the
    library's host IC) and 3 steps with tolerance SOR."""
    from core_collapse_b200.euler2d import ic_random_blob
    p, z = _load("euler2d_random_blob")
    ic = _state(z, "ic")
    _same(ic_random_blob(p).arrays(), ic)
    loop, t, rc = O.eh_main_loop_oracle(p.to_c(), ic, 3, mode=0)
    assert rc == 0 and t == float(z["loop_t"])
    _same(loop, _state(z, "loop"))


def test_fft_golden():
    z = np.load(GOLDEN / "fft.npz")
    for n in (8, 64):
        for inv in (0, 1):
            a = z[f"fft1d_{n}_{inv}_in"].copy()
            O.oracle().or_fft1d(n, O.dp(a), inv)
            assert np.array_equal(a, z[f"fft1d_{n}_{inv}_out"])
    for nx, ny in ((16, 16), (32, 8)):
        p = Params(Nx=nx, Ny=ny, x0=-1, x1=1, y0=-1, y1=1, G=1.0, poisson="fft")
        cp = p.to_c()
        phi = np.zeros(nx * ny)
        O.oracle().or_mhd2d_phi(C.byref(cp), O.dp(z[f"poisson_{nx}x{ny}_rho"].copy()), O.dp(phi), 2, None, None)
        assert np.array_equal(phi, z[f"poisson_{nx}x{ny}_phi"])
