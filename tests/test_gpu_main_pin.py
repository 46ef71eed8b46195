"""The drop-in drivers' output against the reference's own main() (the
compiled reference run once by tests/golden/make_golden.py).

* 2D (cc_mhd2d_main, M2:929-1139), the reference's default parameters
  (192^2, SOR gravity, G = 8): the reference's main() never reaches its HDF5
  write with them (its core collapses near t = 0.275 and dt falls by orders of
  magnitude), so tests/golden/main_mhd2d_log.json holds the lines it printed
  per stored snapshot (t, dt to 7 significant digits, max |div B| to 12) and
  its writer's dataset list.  Checked: max |div B| of the initial state and
  the first snapshot's t and dt as the same strings (the first dt comes from
  the initial state alone, compute_dt M2:579-598); the dataset names, /x /y,
  the (Nt, Ny, Nx) shapes and /t against the printed times; with the
  reference's own lexicographic SOR (--poisson lex) the first printed lines
  string for string; and with the default red-black SOR, stored every 0.01
  up to t = 0.15, dt within a relative MAIN2D_TRAJ_TOL of the reference's at
  the same time (red-black and lexicographic sweeps stop at different
  iterates after a fixed sweep count).
* 3D (cc_mhd3d_main, M3:1132-1338), run to the third stored time: names,
  /x /y /z bit for bit, shapes (Nt, Nz, Ny, Nx), /t[0] within 1e-13, the
  first frame (stored after one step) of every field within 1e-12 of the
  reference's by its sum and maximum (the hybrid EOS's pow runs on the
  device; div B, roundoff itself, relative to |B| / dx) (main_mhd3d.json: its
  HDF5 datasets, recorded in memory)."""
from __future__ import annotations

import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

from core_collapse_b200.mhd2d import Params

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
GOLDEN = ROOT / "tests" / "golden"


def _fixture(name):
    f = GOLDEN / f"main_{name}.json"
    if not f.exists():
        pytest.skip(f"{f.name} not generated")
    return json.loads(f.read_text())


def _values(ent):
    return np.array([float.fromhex(v) for v in ent["values"]])


def _run(exe, *args):
    r = subprocess.run([str(ROOT / "core_collapse_b200" / exe), *map(str, args)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    return r


MAIN2D_TRAJ_TOL = 5e-2
N_LEX_LINES = 10


def _log_fixture():
    f = GOLDEN / "main_mhd2d_log.json"
    if not f.exists():
        pytest.skip(f"{f.name} not generated")
    return json.loads(f.read_text())


def _driver_lines(stdout):
    init, lines = None, []
    for ln in stdout.splitlines():
        if ln.startswith("init max|divB|="):
            init = ln.split("=", 1)[1]
        elif ln.startswith("t="):
            kv = dict(part.split("=", 1) for part in ln.split())
            lines.append([kv["t"], kv["dt"], kv["max|divB|"]])
    return init, lines


def test_mhd2d_driver_first_snapshots_pinned_to_reference_main(tmp_path):
    fx = _log_fixture()
    out = tmp_path / "out"
    init, lines = _driver_lines(_run("cc_mhd2d_main", "--t_end", 0.0045, "--out", out).stdout)
    assert init == fx["init_max_divB"]
    # stores at 1e-3, 2e-3 (one step each), 4e-3 and the clamped last step at t_end
    assert len(lines) == 4 and lines[0][:2] == fx["lines"][0][:2] and lines[-1][0] == "0.0045"
    names = [n.lstrip("/") for n, _ in fx["datasets"]]
    assert sorted(p.stem for p in out.glob("*.npy")) == sorted(names)
    got = {k: np.load(out / f"{k}.npy") for k in names}
    p = Params()
    dx, dy = (p.x1 - p.x0) / p.Nx, (p.y1 - p.y0) / p.Ny
    assert np.array_equal(got["x"], p.x0 + (np.arange(p.Nx) + 0.5) * dx)
    assert np.array_equal(got["y"], p.y0 + (np.arange(p.Ny) + 0.5) * dy)
    nt = len(got["t"])
    assert nt == 5 and got["t"][0] == 0.0
    assert [f"{v:.7g}" for v in got["t"][1:]] == [ln[0] for ln in lines]
    for k in names[3:]:
        assert got[k].shape == (nt, p.Ny, p.Nx), k


def test_mhd2d_driver_lex_prints_the_reference_main_lines(tmp_path):
    """With the reference's own lexicographic SOR (--poisson lex,
    CC_POISSON_SOR_LEX) the driver's state is the reference's to the last bit:
    its printed lines (t, dt, max |div B|) are the reference main's strings."""
    fx = _log_fixture()
    t_end = float(fx["lines"][N_LEX_LINES][0])   # one store more; its step may be clamped to t_end
    init, lines = _driver_lines(_run("cc_mhd2d_main", "--poisson", "lex", "--t_end", t_end, "--out",
                                     tmp_path / "out").stdout)
    assert init == fx["init_max_divB"]
    assert lines[:N_LEX_LINES] == fx["lines"][:N_LEX_LINES]


def test_mhd2d_driver_trajectory_tracks_reference_main(tmp_path):
    """The default red-black SOR: dt at each stored time (every 0.01 up to
    t = 0.15) within MAIN2D_TRAJ_TOL of the reference's dt at the same time
    (interpolated in its printed lines).  Measured: within 2.7% up to t = 0.19;
    beyond, the collapse, whose timing depends on the unconverged 600-sweep
    potential, comes at t = 0.205 with this ordering and near t = 0.275 with
    the reference's (and with --poisson lex)."""
    fx = _log_fixture()
    rt = np.array([float(ln[0]) for ln in fx["lines"]])
    rd = np.array([float(ln[1]) for ln in fx["lines"]])
    r = _run("cc_mhd2d_main", "--dt_store", 0.01, "--t_end", 0.15, "--out", tmp_path / "out")
    _, lines = _driver_lines(r.stdout)
    # the first step (next_store starts at t = 0), t >= 0.01 .. 0.14, and the clamped last step at 0.15
    assert len(lines) == 16 and lines[-1][0] == "0.15"
    worst = 0.0
    for ln in lines[:-1]:
        t, dt = float(ln[0]), float(ln[1])
        worst = max(worst, abs(dt / np.interp(t, rt, rd) - 1.0))
        assert float(ln[2]) < 1e-10, ln
    print(f"max relative difference to the reference main's dt at the same time {worst:.2e}")
    assert worst <= MAIN2D_TRAJ_TOL


def test_mhd3d_driver_output_pinned_to_reference_main(tmp_path):
    fx = _fixture("mhd3d")
    out = tmp_path / "out"
    t_ref = _values(fx["/t"])
    _run("cc_mhd3d_main", "--t_end", float(t_ref[2]), "--out", out)
    names = [k.lstrip("/") for k in fx]
    assert sorted(p.stem for p in out.glob("*.npy")) == sorted(names)
    got = {k: np.load(out / f"{k}.npy") for k in names}
    for k in ("x", "y", "z"):
        assert np.array_equal(got[k], _values(fx["/" + k]))
    nt = len(got["t"])
    assert nt >= 2 and abs(got["t"][0] - t_ref[0]) <= 1e-13 * t_ref[0]
    # div B is roundoff itself: its scale is |B| / dx, not its own size
    bscale = max(fx["/" + b]["frames"][0]["absmax"] for b in ("Bx", "By", "Bz"))
    hmin = min(float(got[a][1] - got[a][0]) for a in ("x", "y", "z"))
    for k in names[4:]:
        ent = fx["/" + k]
        assert list(got[k].shape) == [nt] + ent["dims"][1:], k
        f0 = ent["frames"][0]
        scale = bscale / hmin if k == "divB" else max(f0["absmax"], 1e-300)
        assert abs(float(np.sum(got[k][0])) - f0["sum"]) <= 1e-12 * scale * got[k][0].size, k
        assert abs(float(np.max(np.abs(got[k][0]))) - f0["absmax"]) <= 1e-12 * scale, k


def test_mhd2d_driver_max_steps_ends_the_loop(tmp_path):
    """--max_steps ends the main loop before t_end and keeps what was stored."""
    out = tmp_path / "out"
    r = _run("cc_mhd2d_main", "--max_steps", 3, "--out", out)
    assert "stopped after 3 steps: t=" in r.stdout
    t = np.load(out / "t.npy")
    assert len(t) == 4 and t[0] == 0.0 and np.all(np.diff(t) > 0)   # the t = 0 store and one per step
