"""GPU parity of the 2D Navier-Stokes step (libcc_b200 through its C ABI)
against the CPU oracle (pinned bit for bit to navier_stokes_2d_hllc_poisson.cpp).

Without gravity the FP64 rhs, Heun step and main loop are bit-identical.  With
gravity the spectral solve is the reference's radix-2 transform with its
twiddle recurrence; the one difference is the order of the density-mean sum
(block tree on the GPU, sequential in the reference), which perturbs every
FFT input by at most an ulp of the mean: relative L-inf <= 1e-11 (the
tolerance written in each test).  FP32 tracks the FP64 oracle to relative L1
<= 1e-5 over 10 steps."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_ns2d import CASES_NS, make_case_ns
from core_collapse_b200 import _lib as L
from core_collapse_b200.mhd2d import CcError
from core_collapse_b200.ns2d import DERIVED_NS_FIELDS, Ns2dSolver, ParamsNS, ic_collapse

pytestmark = pytest.mark.gpu

GRAV_TOL = 1e-11


def _tol(p: ParamsNS) -> float:
    return GRAV_TOL if p.gravity_on else 0.0


def _close(got, want, tol, what=""):
    for k, (a, b) in enumerate(zip(got, want)):
        if tol == 0.0:
            assert np.array_equal(a, b), f"{what} field {k}: max |diff| {np.max(np.abs(a - b)):.3e}"
        else:
            r = O.rel_linf(a, b)
            assert r <= tol, f"{what} field {k}: rel L-inf {r:.3e} > {tol:.1e}"


@pytest.mark.parametrize("name", sorted(CASES_NS))
def test_roundtrip_dt_and_rhs(name):
    p, s = make_case_ns(name)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    want_dt = O.oracle().or_ns2d_compute_dt(C.byref(cp), O.pp(S))
    want = O.ns_rhs_oracle(cp, S)
    with Ns2dSolver(p) as g:
        g.upload(s)
        back = g.download()
        assert g.compute_dt() == want_dt
        got = g.compute_rhs()
    for a, b in zip(back.arrays(), S):
        assert np.array_equal(a, b)
    _close(got.arrays(), want, _tol(p), "rhs")


@pytest.mark.parametrize("name", ["collapse_ic", "kicked_viscous", "floors"])
def test_gravity_parity(name):
    p, s = make_case_ns(name)
    cp = p.to_c()
    n = p.Nx * p.Ny
    phi, gx, gy = np.zeros(n), np.zeros(n), np.zeros(n)
    O.oracle().or_ns2d_gravity(C.byref(cp), O.pp(s.arrays()), O.dp(phi), O.dp(gx), O.dp(gy))
    with Ns2dSolver(p) as g:
        g.upload(s)
        got = g.compute_gravity()
    _close(got, [phi, gx, gy], GRAV_TOL, "gravity")


@pytest.mark.parametrize("name", sorted(CASES_NS))
def test_rk2_step_parity(name):
    p, s = make_case_ns(name)
    cp = p.to_c()
    S = [a.copy() for a in s.arrays()]
    dt = O.oracle().or_ns2d_compute_dt(C.byref(cp), O.pp(S))
    want = O.copy_state(S)
    O.oracle().or_ns2d_rk2_step(C.byref(cp), O.pp(want), dt)
    with Ns2dSolver(p) as g:
        g.upload(s)
        g.rk2_step(dt)
        got = g.download()
    _close(got.arrays(), want, _tol(p), "rk2_step")


@pytest.mark.parametrize("name", sorted(CASES_NS))
def test_advance_matches_main_loop(name):
    """cc_ns2d_advance (dt on the device, the loop captured in a CUDA graph
    after the first step) == the main() loop body (NS:758-791), 6 steps."""
    p, s = make_case_ns(name)
    cp = p.to_c()
    want, t_want = O.ns_main_loop_oracle(cp, s.arrays(), 6)
    with Ns2dSolver(p) as g:
        g.upload(s)
        t = g.advance(6, 0.0)
        got = g.download()
        d = g.diagnostics()
    assert d["steps"] == 6 and d["nonfinite"] == 0
    if p.gravity_on:
        assert abs(t - t_want) <= 1e-12 * t_want
    else:
        assert t == t_want
    _close(got.arrays(), want, 10 * _tol(p), "advance")


def test_graph_replay_equals_eager_steps():
    """advance (graph replays) and rk2_step with the dt of compute_dt give the same bits."""
    p, s = make_case_ns("kicked_viscous")
    with Ns2dSolver(p) as a, Ns2dSolver(p) as b:
        a.upload(s)
        b.upload(s)
        a.advance(5)
        for _ in range(5):
            b.rk2_step(b.compute_dt())
        for x, y in zip(a.download().arrays(), b.download().arrays()):
            assert np.array_equal(x, y)


def test_advance_stops_at_t_end():
    p, s = make_case_ns("inviscid_nograv_odd")
    cp = p.to_c()
    dt0 = O.oracle().or_ns2d_compute_dt(C.byref(cp), O.pp([a.copy() for a in s.arrays()]))
    p.t_end = 2.5 * dt0
    with Ns2dSolver(p) as g:
        g.upload(s)
        t = g.advance(10, 0.0)
        steps = g.diagnostics()["steps"]
        assert abs(t - p.t_end) <= 1e-14 and steps <= 4
        before = g.download()
        assert g.advance(3) == t   # past t_end: nothing runs
        after = g.download()
    for x, y in zip(before.arrays(), after.arrays()):
        assert np.array_equal(x, y)
    want, t_want = O.ns_main_loop_oracle(p.to_c(), s.arrays(), 10)
    assert t_want == t
    _close(after.arrays(), want, 0.0, "t_end")


@pytest.mark.parametrize("name", ["collapse_ic", "inviscid_nograv_odd", "floors"])
def test_derived_fields(name):
    p, s = make_case_ns(name)
    cp = p.to_c()
    n = p.Nx * p.Ny
    want = [np.zeros(n) for _ in DERIVED_NS_FIELDS]
    O.oracle().or_ns2d_derived(C.byref(cp), O.pp(s.arrays()), O.pp(want))
    with Ns2dSolver(p) as g:
        g.upload(s)
        got = g.derived()
    for k, w in zip(DERIVED_NS_FIELDS, want):
        a = got[k].ravel()
        if k == "Phi" and p.gravity_on:
            assert O.rel_linf(a, w) <= GRAV_TOL, k
        else:
            assert np.array_equal(a, w), k


def test_fp32_tracks_fp64_oracle():
    p, s = make_case_ns("kicked_viscous")
    want, _ = O.ns_main_loop_oracle(p.to_c(), s.arrays(), 10)
    p32, _ = make_case_ns("kicked_viscous", precision="fp32")
    with Ns2dSolver(p32) as g:
        g.upload(s)
        g.advance(10, 0.0)
        got = g.download()
    for k, (a, b) in enumerate(zip(got.arrays(), want)):
        l1 = np.sum(np.abs(a - b)) / np.sum(np.abs(b))
        assert l1 < 1e-5, f"FP32 field {k}: L1 rel error {l1:.2e}"


def test_reference_ic_runs_and_conserves_mass():
    """The reference's own configuration (NS:54-86 defaults, IC NS:627-689) at
    128^2: 20 steps conserve mass to round-off and stay finite."""
    p = ParamsNS()
    s = ic_collapse(p)
    with Ns2dSolver(p) as g:
        g.upload(s)
        d0 = g.diagnostics()
        g.advance(20, 0.0)
        d1 = g.diagnostics()
    assert d1["nonfinite"] == 0 and d1["steps"] == 20
    assert abs(d1["mass"] - d0["mass"]) <= 1e-13 * d0["mass"]


def test_errors_are_reported():
    with pytest.raises(CcError) as e:
        Ns2dSolver(ParamsNS(Nx=24, Ny=16))   # gravity on needs powers of two
    assert e.value.code == L.CC_ERR_UNSUPPORTED
    p, s = make_case_ns("inviscid_nograv_odd")
    with Ns2dSolver(p) as g:
        with pytest.raises(CcError) as e:
            g.compute_dt()
        assert e.value.code == L.CC_ERR_STATE
        g.upload(s)
        with pytest.raises(CcError) as e:
            g.rk2_step(-1.0)
        assert e.value.code == L.CC_ERR_NONFINITE


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_checkpoint_restart_continues_bitwise(tmp_path, precision):
    """6 steps in one go == 3 steps, checkpoint, load into a fresh handle, 3 more."""
    p, s = make_case_ns("kicked_viscous", precision=precision)
    with Ns2dSolver(p) as g:
        g.upload(s)
        t_full = g.advance(6, 0.0)
        want = g.download()
        steps_full = g.diagnostics()["steps"]
    path = tmp_path / "ck.bin"
    with Ns2dSolver(p) as g:
        g.upload(s)
        g.advance(3, 0.0)
        g.save_checkpoint(path)
    with Ns2dSolver(p) as g:
        g.load_checkpoint(path)
        t = g.advance(3)
        got = g.download()
        d = g.diagnostics()
    assert t == t_full and d["steps"] == steps_full
    for a, w in zip(got.arrays(), want.arrays()):
        assert np.array_equal(a, w)


def test_checkpoint_rejects_bad_files(tmp_path):
    p, s = make_case_ns("kicked_viscous")
    path = tmp_path / "ck.bin"
    with Ns2dSolver(p) as g:
        g.upload(s)
        g.save_checkpoint(path)
    raw = bytearray(path.read_bytes())
    raw[200] ^= 0xFF
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(raw))
    with Ns2dSolver(p) as g:
        for f, code in ((bad, L.CC_ERR_ARG), (tmp_path / "missing.bin", L.CC_ERR_IO)):
            with pytest.raises(CcError) as e:
                g.load_checkpoint(f)
            assert e.value.code == code
    q, _ = make_case_ns("collapse_ic")   # another grid
    with Ns2dSolver(q) as g:
        with pytest.raises(CcError) as e:
            g.load_checkpoint(path)
        assert e.value.code == L.CC_ERR_ARG
    p32, _ = make_case_ns("kicked_viscous", precision="fp32")   # same grid, other precision
    with Ns2dSolver(p32) as g:
        with pytest.raises(CcError) as e:
            g.load_checkpoint(path)
        assert e.value.code == L.CC_ERR_ARG


def test_reference_configuration_runs_to_t_end():
    """The reference main()'s whole run (NS:54-86 defaults: 128^2, t_end 10,
    the collapse IC): about 11 000 Heun steps through cc_ns2d_advance in both
    precisions; the run reaches t_end exactly, stays finite, conserves mass
    (FP64 to round-off), and FP32 and FP64 agree on the density extremes."""
    ext = {}
    for prec in ("fp64", "fp32"):
        p = ParamsNS(precision=prec)
        with Ns2dSolver(p) as g:
            g.upload(ic_collapse(p))
            d0 = g.diagnostics()
            t, chunks = 0.0, 0
            while t < p.t_end - 1e-14 and chunks < 200:
                t = g.advance(1000)
                chunks += 1
            d1 = g.diagnostics()
            rho = g.derived()["rho"]
        assert abs(t - p.t_end) <= 1e-12 and d1["nonfinite"] == 0 and d1["steps"] > 5000
        drift = abs(d1["mass"] - d0["mass"]) / d0["mass"]
        assert drift <= (1e-13 if prec == "fp64" else 1e-6), drift
        ext[prec] = (float(rho.max()), float(rho.min()), d1["steps"])
    assert ext["fp64"][0] > 3.0   # the central condensation has formed
    for k in range(2):
        assert abs(ext["fp32"][k] - ext["fp64"][k]) <= 1e-3 * ext["fp64"][k]
