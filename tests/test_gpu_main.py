"""The drop-in 2D driver cc_mhd2d_main (the reference main(),
mhd2d_resistive_hlld_ct_gravity.cpp:928-1130): its snapshots against the same
loop driven through the Python wrapper, its output files, and restart from its
checkpoint."""
from __future__ import annotations

import subprocess
from pathlib import Path

import numpy as np
import pytest

from core_collapse_b200.mhd2d import DERIVED_FIELDS, Mhd2dSolver, Params, ic_reference

pytestmark = pytest.mark.gpu

EXE = Path(__file__).resolve().parent.parent / "core_collapse_b200" / "cc_mhd2d_main"
N, T_END, DT_STORE = 32, 0.004, 0.0015


def _run(*args) -> str:
    r = subprocess.run([str(EXE), *map(str, args)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _load(out: Path) -> dict:
    return {k: np.load(out / f"{k}.npy") for k in ("x", "y", "t", *DERIVED_FIELDS)}


def test_main_matches_wrapper_loop(tmp_path):
    out = tmp_path / "out"
    log = _run("--Nx", N, "--Ny", N, "--t_end", T_END, "--dt_store", DT_STORE, "--out", out)
    assert log.startswith("init max|divB|=")
    got = _load(out)
    # the same loop through the Python wrapper (defaults, reference IC, store rule)
    p = Params(Nx=N, Ny=N, t_end=T_END, dt_store=DT_STORE)
    U, B = ic_reference(p)
    ts, snaps = [0.0], []
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        snaps.append(s.derived())
        t, next_store = 0.0, 0.0
        while t < p.t_end:
            t = s.advance(1)
            if t >= next_store - 1e-15:
                ts.append(t)
                snaps.append(s.derived())
                next_store += p.dt_store
    assert np.array_equal(got["t"], np.array(ts))
    assert got["x"].shape == (N,) and got["y"].shape == (N,)
    assert np.allclose(got["x"], p.x0 + (np.arange(N) + 0.5) * (p.x1 - p.x0) / N, rtol=0, atol=1e-15)
    for k in DERIVED_FIELDS:
        assert got[k].shape == (len(ts), N, N)
        for n, snap in enumerate(snaps):
            assert np.array_equal(got[k][n], snap[k]), f"{k} snapshot {n}"


def test_main_restart_continues_from_checkpoint(tmp_path):
    """A run that writes a checkpoint at its end, then a run restarted from it:
    the restarted run's first snapshot is the checkpointed state at its time."""
    ck = tmp_path / "ck.bin"
    a, b = tmp_path / "a", tmp_path / "b"
    _run("--Nx", N, "--Ny", N, "--t_end", T_END, "--dt_store", DT_STORE, "--out", a, "--checkpoint", ck)
    _run("--Nx", N, "--Ny", N, "--t_end", 2 * T_END, "--dt_store", DT_STORE, "--out", b, "--restart", ck)
    A, B = _load(a), _load(b)
    p = Params(Nx=N, Ny=N, t_end=2 * T_END, dt_store=DT_STORE)
    with Mhd2dSolver(p) as s:
        s.load_checkpoint(ck)
        t_ck = s.diagnostics()["t"]
        want = s.derived()
    assert B["t"][0] == t_ck and abs(t_ck - T_END) < 1e-12 and A["t"][-1] <= t_ck
    assert B["t"][-1] <= 2 * T_END and len(B["t"]) >= 2
    for k in DERIVED_FIELDS:
        assert np.array_equal(B[k][0], want[k]), k


EXE_EH = EXE.parent / "cc_euler2d_main"


def test_euler_main_matches_wrapper_loop(tmp_path):
    """cc_euler2d_main (the reference main() of euler2d_gravity_hllc.cpp,
    EH:645-737): its snapshots equal the same loop driven through the Python
    wrapper, bit for bit."""
    from core_collapse_b200.euler2d import Euler2dSolver, ParamsEH, ic_random_blob
    out = tmp_path / "eh"
    r = subprocess.run([str(EXE_EH), "--Nx", "32", "--Ny", "32", "--t_end", "0.01", "--dt_store", "0.004",
                        "--out", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = {k: np.load(out / f"{k}.npy") for k in ("x", "y", "t", "rho", "P", "Mach")}
    p = ParamsEH(Nx=32, Ny=32, t_end=0.01, dt_store=0.004)
    ts, snaps = [0.0], []
    with Euler2dSolver(p) as s:
        s.upload(ic_random_blob(p))
        snaps.append(s.derived())
        t, next_store = 0.0, p.dt_store
        while t < p.t_end - 1e-14:
            t = s.advance(1)
            if t + 1e-14 >= next_store or t >= p.t_end - 1e-14:
                ts.append(t)
                snaps.append(s.derived())
                next_store += p.dt_store
    assert np.array_equal(got["t"], np.array(ts)) and got["x"].shape == (32,)
    for k in ("rho", "P", "Mach"):
        assert got[k].shape == (len(ts), 32, 32)
        for n, snap in enumerate(snaps):
            assert np.array_equal(got[k][n], snap[k]), f"{k} snapshot {n}"


EXE_3D = EXE.parent / "cc_mhd3d_main"


def test_mhd3d_main_matches_wrapper_loop(tmp_path):
    """cc_mhd3d_main (the reference main() of mhd3d_resistive_hlld_ct.cpp): the
    reference IC, the loop and its store rule (no frame at t = 0); snapshots equal
    the same loop driven through the Python wrapper, bit for bit."""
    from core_collapse_b200.mhd3d import DERIVED3_FIELDS, Mhd3dSolver, Params3, ic_reference3
    out = tmp_path / "m3"
    n, t_end, dts = 16, 0.004, 0.0015
    r = subprocess.run([str(EXE_3D), "--Nx", str(n), "--Ny", str(n), "--Nz", str(n), "--t_end", str(t_end),
                        "--dt_store", str(dts), "--out", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = {k: np.load(out / f"{k}.npy") for k in ("x", "y", "z", "t", *DERIVED3_FIELDS)}
    p = Params3(Nx=n, Ny=n, Nz=n, t_end=t_end, dt_store=dts)
    ts, snaps = [], []
    with Mhd3dSolver(p) as s:
        s.upload(ic_reference3(p))
        t, tnext = 0.0, 0.0
        while t < p.t_end:
            t = s.advance(1)
            if t >= tnext - 1e-12:
                ts.append(t)
                snaps.append(s.derived())
                tnext += p.dt_store
    assert np.array_equal(got["t"], np.array(ts)) and got["z"].shape == (n,)
    for k in DERIVED3_FIELDS:
        assert got[k].shape == (len(ts), n, n, n)
        for m, snap in enumerate(snaps):
            assert np.array_equal(got[k][m], snap[k]), f"{k} snapshot {m}"


EXE_NS = EXE.parent / "cc_ns2d_main"


def test_ns2d_main_matches_wrapper_loop(tmp_path):
    """cc_ns2d_main (the reference main() of navier_stokes_2d_hllc_poisson.cpp,
    NS:611-803): the reference IC, loop and store rule (frame at t = 0);
    snapshots equal the same loop driven through the Python wrapper, bit for bit."""
    from core_collapse_b200.ns2d import DERIVED_NS_FIELDS, Ns2dSolver, ParamsNS, ic_collapse
    out = tmp_path / "ns"
    n, t_end, dts = 32, 0.05, 0.02
    r = subprocess.run([str(EXE_NS), "--Nx", str(n), "--Ny", str(n), "--t_end", str(t_end), "--dt_store", str(dts),
                        "--out", str(out)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    got = {k: np.load(out / f"{k}.npy") for k in ("x", "y", "t", *DERIVED_NS_FIELDS)}
    p = ParamsNS(Nx=n, Ny=n, t_end=t_end, dt_store=dts)
    ts, snaps = [0.0], []
    with Ns2dSolver(p) as s:
        s.upload(ic_collapse(p))
        snaps.append(s.derived())
        t, next_store = 0.0, p.dt_store
        while t < p.t_end - 1e-14:
            t = s.advance(1)
            if t + 1e-14 >= next_store or t >= p.t_end - 1e-14:
                ts.append(t)
                snaps.append(s.derived())
                next_store += p.dt_store
    assert len(ts) >= 3 and np.array_equal(got["t"], np.array(ts)) and got["x"].shape == (n,)
    for k in DERIVED_NS_FIELDS:
        assert got[k].shape == (len(ts), n, n)
        for m, snap in enumerate(snaps):
            assert np.array_equal(got[k][m], snap[k]), f"{k} snapshot {m}"


@pytest.mark.parametrize("exe,mod", [("cc_ns2d_main", "ns2d"), ("cc_euler2d_main", "euler2d")])
def test_2d_drivers_restart_from_checkpoint(tmp_path, exe, mod):
    """--checkpoint at the end of one run, --restart of a longer one: the
    restarted run's first snapshot is the checkpointed state at its time and it
    ends at the same t_end as an uninterrupted run (whose trajectory differs:
    the first run's last step was clamped to its own t_end)."""
    import importlib
    m = importlib.import_module(f"core_collapse_b200.{mod}")
    Solver = m.Ns2dSolver if mod == "ns2d" else m.Euler2dSolver
    Par = m.ParamsNS if mod == "ns2d" else m.ParamsEH
    fields = m.DERIVED_NS_FIELDS if mod == "ns2d" else ("rho", "P", "Mach")
    prog = EXE.parent / exe
    n, t1, t2, dts = 32, 0.02, 0.04, 0.01
    ck, a, b, full = tmp_path / "ck.bin", tmp_path / "a", tmp_path / "b", tmp_path / "full"
    common = ["--Nx", n, "--Ny", n, "--dt_store", dts]
    for args in ([*common, "--t_end", t1, "--out", a, "--checkpoint", ck],
                 [*common, "--t_end", t2, "--out", b, "--restart", ck],
                 [*common, "--t_end", t2, "--out", full]):
        r = subprocess.run([str(prog), *map(str, args)], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
    A, B, F = ({k: np.load(d / f"{k}.npy") for k in ("t", *fields)} for d in (a, b, full))
    with Solver(Par(Nx=n, Ny=n)) as s:
        s.load_checkpoint(ck)
        t_ck = s.diagnostics()["t"]
        want = s.derived()
    assert B["t"][0] == t_ck == A["t"][-1] and abs(t_ck - t1) < 1e-12
    assert B["t"][-1] == F["t"][-1]
    for k in fields:
        assert np.array_equal(B[k][0], want[k]), k
        assert B[k].shape[1:] == F[k].shape[1:]
