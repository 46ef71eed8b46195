"""GPU parity of the 2D MHD step (libcc_b200 through its C ABI) against the CPU
oracle on the same seeded inputs.

Tolerance: FP64 relative L-inf per field, max|gpu - oracle| / max|oracle|,
<= 1e-12.  The FP64 kernels are built with -fmad=false and keep the
reference's operation order, so without gravity the step is bit-identical;
with gravity the only differences come from the density/potential mean sums,
which the GPU reduces as a fixed tree instead of the reference's sequential
loop (~1e-16 relative).  The FP32 path is checked against the FP64 oracle with
a loose bound and its error is reported."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O
from cases_mhd2d import CASES, make_case
from core_collapse_b200 import _lib as L
from core_collapse_b200.mhd2d import GravField, Mhd2dSolver, Params, CcError, ic_orszag_tang, ic_collapse

pytestmark = pytest.mark.gpu

TOL = 1e-12
FIELDS = ["rho", "mx", "my", "mz", "E", "Bz", "Bx_f", "By_f"]


def _assert_close(got, want, tol=TOL, what=""):
    for k, (a, b) in enumerate(zip(got, want)):
        r = O.rel_linf(a, b)
        assert r <= tol, f"{what} field {FIELDS[k]}: rel L-inf {r:.3e} > {tol:.1e}"


def _gpu_state(s: Mhd2dSolver):
    U, B = s.download()
    return O.state_list(U, B)


@pytest.mark.parametrize("name", sorted(CASES))
def test_upload_download_roundtrip(name):
    p, U, B = make_case(name)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        got = _gpu_state(s)
    for a, b in zip(got, O.state_list(U, B)):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("name", sorted(CASES))
def test_compute_dt_bitwise(name):
    p, U, B = make_case(name)
    cp = p.to_c()
    want = O.oracle().or_mhd2d_compute_dt(C.byref(cp), O.pp(O.state_list(U, B)))
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        assert s.compute_dt() == want


@pytest.mark.parametrize("name", sorted(CASES))
def test_rk2_step_parity(name):
    """rk2_step with host gravity for stage 1 and the device red-black SOR for
    stage 2, against the oracle's rk2_step with the same SOR ordering."""
    p, U, B = make_case(name)
    cp = p.to_c()
    S = O.state_list(U, B)
    gx, gy, _, _ = O.m2_gravity_oracle(cp, U.rho, mode=1)
    dt = O.oracle().or_mhd2d_compute_dt(C.byref(cp), O.pp(S))
    want = O.m2_rk2_oracle(cp, S, gx, gy, dt, mode=1)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        s.rk2_step(GravField(gx, gy), dt)
        got = _gpu_state(s)
    if not p.gravity_on:
        for k, (a, b) in enumerate(zip(got, want)):
            assert np.array_equal(a, b), f"field {FIELDS[k]} not bit-identical without gravity"
    _assert_close(got, want, what=name)


@pytest.mark.parametrize("name", [n for n in sorted(CASES) if CASES[n][0].get("gravity_on")])
def test_gravity_sor_parity(name):
    p, U, B = make_case(name)
    cp = p.to_c()
    gx, gy, it, res = O.m2_gravity_oracle(cp, U.rho, mode=1)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        g = s.compute_gravity()
        d = s.diagnostics()
    assert d["poisson_iters"] == it
    assert O.rel_linf(g.gx, gx) <= TOL and O.rel_linf(g.gy, gy) <= TOL


def test_gravity_sor_tolerance_stops_like_oracle():
    p, U, B = make_case("periodic_grav_eta")
    p.sor_tol = 1e-9
    p.sor_iters = 100000
    cp = p.to_c()
    gx, gy, it, res = O.m2_gravity_oracle(cp, U.rho, mode=1)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        g = s.compute_gravity()
        d = s.diagnostics()
    assert abs(d["poisson_iters"] - it) <= 2
    assert d["poisson_residual"] < 1e-9
    assert O.rel_linf(g.gx, gx) <= 1e-9 and O.rel_linf(g.gy, gy) <= 1e-9


@pytest.mark.parametrize("shape", [(16, 16), (32, 8), (8, 64), (128, 64)])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_gravity_fft_parity(shape, precision):
    nx, ny = shape
    p = Params(Nx=nx, Ny=ny, x0=-1, x1=1, y0=-1, y1=1, G=1.0, poisson="fft", precision=precision,
               gravity_on=True)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.2)
    cp = p.to_c()
    gx, gy, _, _ = O.m2_gravity_oracle(cp, U.rho, mode=2)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        g = s.compute_gravity()
    tol = TOL if precision == "fp64" else 2e-5
    assert O.rel_linf(g.gx, gx) <= tol and O.rel_linf(g.gy, gy) <= tol


@pytest.mark.parametrize("name,poisson", [("periodic_grav_eta", "sor"), ("outflow_grav_eta", "sor"),
                                          ("mixed_ot_ideal", "sor"), ("reference_ic", "sor")])
def test_advance_matches_main_loop(name, poisson):
    """cc_mhd2d_advance (device loop, dt on the device) == the main() loop body."""
    p, U, B = make_case(name, poisson=poisson)
    p.t_end = 10.0
    cp = p.to_c()
    want, t_want = O.m2_main_loop_oracle(cp, O.state_list(U, B), 6, mode=1)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        t = s.advance(6, 0.0)
        got = _gpu_state(s)
        d = s.diagnostics()
    assert d["steps"] == 6
    assert abs(t - t_want) <= 1e-12 * t_want
    _assert_close(got, want, what=name)


def test_advance_fft_graph_matches_main_loop():
    """Periodic FFT gravity: the captured-graph path (3-step graphs) plus eager
    remainder steps against the oracle's spectral main loop."""
    p = Params(Nx=64, Ny=32, x0=-1, x1=1, y0=-1, y1=1, eta=1e-3, G=1.0, gravity_on=True, poisson="fft", cfl=0.4,
               t_end=10.0)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.2)
    cp = p.to_c()
    want, t_want = O.m2_main_loop_oracle(cp, O.state_list(U, B), 8, mode=2)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        t = s.advance(8, 0.0)
        got = _gpu_state(s)
    assert abs(t - t_want) <= 1e-12 * t_want
    _assert_close(got, want, what="fft")


def test_advance_gravity_off_bit_identical():
    p, U, B = make_case("mixed_ot_ideal")
    p.t_end = 10.0
    cp = p.to_c()
    want, t_want = O.m2_main_loop_oracle(cp, O.state_list(U, B), 7, mode=1)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        t = s.advance(7, 0.0)
        got = _gpu_state(s)
    assert t == t_want
    for k, (a, b) in enumerate(zip(got, want)):
        assert np.array_equal(a, b), f"field {FIELDS[k]}"


def test_advance_stops_at_t_end():
    p, U, B = make_case("mixed_ot_ideal")
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        dt0 = s.compute_dt()
        p_end = 2.5 * dt0
    p.t_end = p_end
    cp = p.to_c()
    want, t_want = O.m2_main_loop_oracle(cp, O.state_list(U, B), 10, mode=1)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        t = s.advance(10, 0.0)
        got = _gpu_state(s)
        d = s.diagnostics()
    assert t == p_end == t_want
    assert 2 <= d["steps"] <= 4
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


def test_divB_stays_at_roundoff_and_mass_conserved():
    p = Params(Nx=64, Ny=64, x0=-1, x1=1, y0=-1, y1=1, eta=1e-3, gravity_on=True, G=1.0, poisson="fft", cfl=0.4,
               t_end=10.0)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.2)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        d0 = s.diagnostics()
        s.advance(30, 0.0)
        d1 = s.diagnostics()
    bscale = 1.0 / np.sqrt(4 * np.pi) / p.dx
    assert d0["max_divB"] < 1e-12 * bscale
    assert d1["max_divB"] < 1e-11 * bscale
    assert abs(d1["mass"] - d0["mass"]) <= 1e-13 * d0["mass"]


def test_energy_conserved_ideal_periodic():
    """eta = 0, no gravity, periodic, no floor activity: total energy and
    momentum change only by roundoff (flux-form update)."""
    p = Params(Nx=64, Ny=64, x0=-1, x1=1, y0=-1, y1=1, eta=0.0, gravity_on=False, cfl=0.4, t_end=10.0)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.2)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        d0 = s.diagnostics()
        s.advance(20, 0.0)
        d1 = s.diagnostics()
    assert abs(d1["energy"] - d0["energy"]) <= 1e-12 * abs(d0["energy"])
    assert abs(d1["mass"] - d0["mass"]) <= 1e-13 * d0["mass"]
    assert abs(d1["mom_x"] - d0["mom_x"]) <= 1e-12 * (abs(d0["mom_x"]) + d0["mass"])


def test_fp32_path_tracks_fp64_oracle():
    p = Params(Nx=64, Ny=64, x0=-1, x1=1, y0=-1, y1=1, eta=1e-3, gravity_on=True, G=1.0, poisson="fft", cfl=0.4,
               t_end=10.0)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.2)
    want, _ = O.m2_main_loop_oracle(p.to_c(), O.state_list(U, B), 10, mode=2)
    p32 = Params(**{**p.__dict__, "precision": "fp32"})
    with Mhd2dSolver(p32) as s:
        s.upload(U, B)
        s.advance(10, 0.0)
        got = _gpu_state(s)
    for k, (a, b) in enumerate(zip(got, want)):
        den = np.sum(np.abs(b))
        if den == 0.0:
            assert np.max(np.abs(a)) == 0.0, f"FP32 field {FIELDS[k]} should stay zero"
            continue
        l1 = np.sum(np.abs(a - b)) / den
        assert l1 < 1e-5, f"FP32 field {FIELDS[k]} L1 rel error {l1:.2e}"


def test_errors_are_reported():
    p = Params(Nx=12, Ny=10, poisson="fft")
    with pytest.raises(CcError) as e:
        Mhd2dSolver(p)
    assert e.value.code == L.CC_ERR_UNSUPPORTED
    p, U, B = make_case("periodic_grav_eta")
    with Mhd2dSolver(p) as s:
        with pytest.raises(CcError) as e:
            s.rk2_step(None, 1e-3)     # no state uploaded
        assert e.value.code == L.CC_ERR_STATE
        s.upload(U, B)
        with pytest.raises(CcError) as e:
            s.rk2_step(None, 1e-3)     # no device gravity computed for this state
        assert e.value.code == L.CC_ERR_STATE
        with pytest.raises(CcError) as e:
            s.rk2_step(None, float("nan"))
        assert e.value.code == L.CC_ERR_NONFINITE


@pytest.mark.parametrize("name", sorted(CASES))
def test_derived_fields_match_oracle(name):
    """cc_mhd2d_derived == the reference main()'s snapshot store (M2:1065-1106)
    bit for bit in FP64, after 3 steps so that every field is non-trivial."""
    p, U, B = make_case(name)
    p.t_end = 10.0
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        s.advance(3, 0.0)
        got = s.derived()
        S = _gpu_state(s)
    want = O.m2_derived_oracle(p.to_c(), S)
    from core_collapse_b200.mhd2d import DERIVED_FIELDS
    for k, name_k in enumerate(DERIVED_FIELDS):
        assert np.array_equal(got[name_k].ravel(), want[k]), f"{name} field {name_k}"


def test_derived_fields_fp32_close():
    p, U, B = make_case("periodic_grav_eta", precision="fp32")
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        got = s.derived()
        S = _gpu_state(s)
    want = O.m2_derived_oracle(p.to_c(), S)
    from core_collapse_b200.mhd2d import DERIVED_FIELDS
    for k, name_k in enumerate(DERIVED_FIELDS[:9]):
        scale = np.max(np.abs(want[k])) + 1e-30
        assert np.max(np.abs(got[name_k].ravel() - want[k])) <= 1e-5 * scale, name_k
    assert np.max(np.abs(got["divB"])) < 1e-4


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_checkpoint_restart_continues_bitwise(tmp_path, precision):
    """6 steps in one go == 3 steps, checkpoint, load into a fresh handle, 3
    more steps: state, time and step count identical."""
    p, U, B = make_case("periodic_grav_eta", precision=precision)
    p.t_end = 10.0
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        t_full = s.advance(6, 0.0)
        want = _gpu_state(s)
        steps_full = s.diagnostics()["steps"]
    path = tmp_path / "ck.bin"
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        s.advance(3, 0.0)
        s.save_checkpoint(path)
    with Mhd2dSolver(p) as s:
        s.load_checkpoint(path)
        t = s.advance(3)
        got = _gpu_state(s)
        d = s.diagnostics()
    assert t == t_full and d["steps"] == steps_full
    for a, w in zip(got, want):
        assert np.array_equal(a, w)


def test_checkpoint_rejects_bad_files(tmp_path):
    p, U, B = make_case("periodic_grav_eta")
    path = tmp_path / "ck.bin"
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        s.save_checkpoint(path)
    raw = bytearray(path.read_bytes())
    raw[100] ^= 0xFF
    bad = tmp_path / "bad.bin"
    bad.write_bytes(bytes(raw))
    q, U2, B2 = make_case("outflow_grav_eta")
    with Mhd2dSolver(p) as s:
        with pytest.raises(CcError) as e:
            s.load_checkpoint(bad)
        assert e.value.code == L.CC_ERR_ARG
        with pytest.raises(CcError) as e:
            s.load_checkpoint(tmp_path / "missing.bin")
        assert e.value.code == L.CC_ERR_IO
    with Mhd2dSolver(q) as s:
        with pytest.raises(CcError) as e:
            s.load_checkpoint(path)
        assert e.value.code == L.CC_ERR_ARG
