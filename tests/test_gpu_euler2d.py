"""GPU parity of the 2D Euler/HLLC step (libcc_b200 through its C ABI)
against the CPU oracle (pinned bit-for-bit to euler2d_gravity_hllc.cpp).

Without gravity the FP64 step is bit-identical.  With gravity the GPU runs
red-black SOR (the oracle's red-black restatement is the reference): with a
fixed sweep count the only difference is the FP64 mean-reduction order
(relative L-inf <= 1e-12); with the residual tolerance the stopping sweep may
differ by one or two, bounded by the tolerance (<= 1e-8)."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_euler2d import CASES_EH, make_case_eh
from core_collapse_b200 import _lib as L
from core_collapse_b200.euler2d import Euler2dSolver, ParamsEH, ic_random_blob
from core_collapse_b200.mhd2d import CcError

pytestmark = pytest.mark.gpu


def _fixed_sweeps(p: ParamsEH, n=150):
    p.sor_tol = 0.0
    p.sor_max_iter = n
    return p


def _close(got, want, tol):
    for k, (a, b) in enumerate(zip(got, want)):
        r = O.rel_linf(a, b)
        assert r <= tol, f"field {k}: rel L-inf {r:.3e} > {tol:.1e}"


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_roundtrip_and_dt_bitwise(name):
    p, s = make_case_eh(name)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    want = O.oracle().or_euler2d_compute_dt(C.byref(cp), O.pp(S))
    with Euler2dSolver(p) as g:
        g.upload(s)
        got = g.download()
        assert g.compute_dt() == want
    for a, b in zip(got.arrays(), S):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_rk2_step_parity(name):
    p, s = make_case_eh(name)
    _fixed_sweeps(p)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    dt = O.oracle().or_euler2d_compute_dt(C.byref(cp), O.pp(S))
    want = O.copy_state(S)
    O.oracle().or_euler2d_rk2_step(C.byref(cp), O.pp(want), dt, 1)
    with Euler2dSolver(p) as g:
        g.upload(s)
        g.rk2_step(dt)
        got = g.download().arrays()
    if not p.gravity_on:
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
    _close(got, want, 1e-12)


def test_gravity_with_tolerance_matches_red_black_oracle():
    p, s = make_case_eh("periodic_grav")
    cp = p.to_c()
    n = p.Nx * p.Ny
    gx, gy = np.zeros(n), np.zeros(n)
    it, res = C.c_int(), C.c_double()
    O.oracle().or_euler2d_gravity(C.byref(cp), O.dp(s.rho), O.dp(gx), O.dp(gy), 1, C.byref(it), C.byref(res))
    with Euler2dSolver(p) as g:
        g.upload(s)
        x, y = g.compute_gravity()
        d = g.diagnostics()
    assert abs(d["poisson_iters"] - it.value) <= 2 and d["poisson_residual"] < p.sor_tol
    assert O.rel_linf(x, gx) <= 1e-8 and O.rel_linf(y, gy) <= 1e-8


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_advance_matches_main_loop(name):
    p, s = make_case_eh(name)
    _fixed_sweeps(p)
    p.t_end = 10.0
    cp = p.to_c()
    want, t_want, rc = O.eh_main_loop_oracle(cp, [a.copy() for a in s.arrays()], 4, mode=1)
    assert rc == 0
    with Euler2dSolver(p) as g:
        g.upload(s)
        t = g.advance(4, 0.0)
        got = g.download().arrays()
        d = g.diagnostics()
    assert d["steps"] == 4
    if not p.gravity_on:
        assert t == t_want
        for a, b in zip(got, want):
            assert np.array_equal(a, b)
    else:
        assert abs(t - t_want) <= 1e-12 * t_want
        _close(got, want, 1e-12)


def test_reference_ic_loop_and_mass():
    """The reference's own main(): random-blob IC, SOR to 1e-10, 3 steps;
    mass (periodic, floors idle) conserved to roundoff."""
    p = ParamsEH(Nx=32, Ny=32, t_end=10.0)
    U = ic_random_blob(p)
    cp = p.to_c()
    want, t_want, rc = O.eh_main_loop_oracle(cp, [a.copy() for a in U.arrays()], 3, mode=1)
    with Euler2dSolver(p) as g:
        g.upload(U)
        d0 = g.diagnostics()
        t = g.advance(3, 0.0)
        d1 = g.diagnostics()
        got = g.download().arrays()
    assert abs(t - t_want) <= 1e-9 * t_want
    _close(got, want, 1e-8)
    assert abs(d1["mass"] - d0["mass"]) <= 1e-13 * d0["mass"]


def test_bad_dt_stops_the_loop():
    """An infinite momentum makes dt = 0: the reference aborts (EH:699-702),
    the device loop stops with CC_ERR_NONFINITE and keeps the last good state."""
    p, s = make_case_eh("mixed_nograv")
    s.mx[5] = np.inf
    p.t_end = 10.0
    rc_or = O.eh_main_loop_oracle(p.to_c(), [a.copy() for a in s.arrays()], 3, mode=1)[2]
    assert rc_or == L.CC_ERR_NONFINITE
    with Euler2dSolver(p) as g:
        g.upload(s)
        with pytest.raises(CcError) as e:
            g.advance(3, 0.0)
        assert e.value.code == L.CC_ERR_NONFINITE
        d = g.diagnostics()
        assert d["steps"] == 0
        back = g.download()
    assert np.array_equal(back.rho, s.rho)


def test_odd_extent_with_gravity_is_rejected():
    """The red-black SOR colouring needs even extents on its (always periodic)
    axes; an odd grid with gravity is refused at create time, not mis-solved."""
    p, _ = make_case_eh("outflow_odd_nograv")
    p.gravity_on = True
    with pytest.raises(CcError) as e:
        Euler2dSolver(p)
    assert e.value.code == L.CC_ERR_UNSUPPORTED


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_derived_fields_match_oracle(name):
    """cc_euler2d_derived == the reference main()'s snapshot store (EH:661-689)
    bit for bit in FP64; the cases hold cold cells, so the floors act."""
    p, s = make_case_eh(name)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    n = p.Nx * p.Ny
    want = [np.empty(n) for _ in range(3)]
    O.oracle().or_euler2d_derived(C.byref(cp), O.pp(S), O.pp(want))
    with Euler2dSolver(p) as g:
        g.upload(s)
        got = g.derived()
    for k, name_k in enumerate(("rho", "P", "Mach")):
        assert np.array_equal(got[name_k].ravel(), want[k]), f"{name} {name_k}"


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_enclosed_mass_gravity_matches_oracle(name):
    """poisson="enclosed" (compute_enclosed_mass_gravity, EH:226-286, the rhs's
    commented-out alternative): gravity, one RK2 step and 5 steps of the main
    loop against the oracle restatement (itself bit-identical to the compiled
    reference); the GPU scan sums in another association, so 1e-12."""
    p, s = make_case_eh(name)
    p.gravity_on, p.poisson = True, "enclosed"
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    n = p.Nx * p.Ny
    wx, wy = np.zeros(n), np.zeros(n)
    O.oracle().or_euler2d_gravity(C.byref(cp), O.dp(S[0]), O.dp(wx), O.dp(wy), 0, None, None)
    dt = O.oracle().or_euler2d_compute_dt(C.byref(cp), O.pp(S))
    want = O.copy_state(S)
    O.oracle().or_euler2d_rk2_step(C.byref(cp), O.pp(want), dt, 1)
    p.t_end = 10.0
    want5, _, _ = O.eh_main_loop_oracle(p.to_c(), O.copy_state(S), 5, mode=1)
    with Euler2dSolver(p) as g:
        g.upload(s)
        gx, gy = g.compute_gravity()
        g.rk2_step(dt)
        got = g.download().arrays()
    with Euler2dSolver(p) as g:
        g.upload(s)
        g.advance(5, 0.0)
        got5 = g.download().arrays()
    assert O.rel_linf(gx, wx) <= 1e-12 and O.rel_linf(gy, wy) <= 1e-12
    for a, b in zip(got, want):
        assert O.rel_linf(a, b) <= 1e-12
    for a, b in zip(got5, want5):
        assert O.rel_linf(a, b) <= 1e-11


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_checkpoint_restart_continues_bitwise(tmp_path, precision):
    """6 steps in one go == 3 steps, checkpoint, load into a fresh handle, 3 more
    (SOR gravity, so the restart also carries the Poisson state's effect)."""
    p, s = make_case_eh("periodic_grav")
    p.precision = precision
    with Euler2dSolver(p) as g:
        g.upload(s)
        t_full = g.advance(6, 0.0)
        want = g.download()
        steps_full = g.diagnostics()["steps"]
    path = tmp_path / "ck.bin"
    with Euler2dSolver(p) as g:
        g.upload(s)
        g.advance(3, 0.0)
        g.save_checkpoint(path)
    with Euler2dSolver(p) as g:
        g.load_checkpoint(path)
        t = g.advance(3)
        got = g.download()
        d = g.diagnostics()
    assert t == t_full and d["steps"] == steps_full
    for a, w in zip(got.arrays(), want.arrays()):
        assert np.array_equal(a, w)


def test_checkpoint_rejects_bad_files(tmp_path):
    p, s = make_case_eh("periodic_grav")
    path = tmp_path / "ck.bin"
    with Euler2dSolver(p) as g:
        g.upload(s)
        g.save_checkpoint(path)
    raw = bytearray(path.read_bytes())
    raw[-20] ^= 0x01
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(raw))
    with Euler2dSolver(p) as g:
        with pytest.raises(CcError) as e:
            g.load_checkpoint(bad)
        assert e.value.code == L.CC_ERR_ARG
    q, _ = make_case_eh("outflow_grav")   # other boundaries
    with Euler2dSolver(q) as g:
        with pytest.raises(CcError) as e:
            g.load_checkpoint(path)
        assert e.value.code == L.CC_ERR_ARG


@pytest.mark.parametrize("name", sorted(CASES_EH))
def test_shell_gravity_matches_oracle(name):
    """poisson="shells" (gravity_accel_from_enclosed_mass, gravity_enclosed.h:18-96):
    gravity, one RK2 step and 5 steps of the main loop against the oracle
    restatement (bit-identical to the compiled header); the GPU scan sums the
    shell masses in another association, so 1e-12."""
    p, s = make_case_eh(name)
    p.gravity_on, p.poisson, p.Nr_bins, p.xc, p.yc = True, "shells", 24, 0.45, 0.55
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    n = p.Nx * p.Ny
    wx, wy = np.zeros(n), np.zeros(n)
    O.oracle().or_euler2d_gravity(C.byref(cp), O.dp(S[0]), O.dp(wx), O.dp(wy), 0, None, None)
    dt = O.oracle().or_euler2d_compute_dt(C.byref(cp), O.pp(S))
    want = O.copy_state(S)
    O.oracle().or_euler2d_rk2_step(C.byref(cp), O.pp(want), dt, 1)
    p.t_end = 10.0
    want5, _, _ = O.eh_main_loop_oracle(p.to_c(), O.copy_state(S), 5, mode=1)
    with Euler2dSolver(p) as g:
        g.upload(s)
        gx, gy = g.compute_gravity()
        g.rk2_step(dt)
        got = g.download().arrays()
    with Euler2dSolver(p) as g:
        g.upload(s)
        g.advance(5, 0.0)
        got5 = g.download().arrays()
    assert O.rel_linf(gx, wx) <= 1e-12 and O.rel_linf(gy, wy) <= 1e-12
    for a, b in zip(got, want):
        assert O.rel_linf(a, b) <= 1e-12
    for a, b in zip(got5, want5):
        assert O.rel_linf(a, b) <= 1e-11
