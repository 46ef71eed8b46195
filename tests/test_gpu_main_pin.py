"""The drop-in drivers' output against what the reference's own main() wrote
(tests/golden/main_mhd2d.json, main_mhd3d.json: its HDF5 datasets, recorded by
running the compiled reference once; see tests/golden/make_golden.py).

The drivers write each dataset as <name>.npy.  Checked, with the reference's
default parameters:
* 2D (cc_mhd2d_main, M2:929-1139), run to t_end = 0.02: the dataset names
  are the reference's; /x, /y bit for bit; each field's shape is
  (Nt, Ny, Nx); the t = 0 frame of every field bit for bit (SHA-256 of the FP64
  values); /t[0], /t[1] bit for bit (the first dt comes from the initial state
  through compute_dt, M2:579-598); the later stored times within 1e-9 of the
  reference's (the driver's red-black SOR and the reference's lexicographic
  sweeps stop at different iterates, which moves dt in its last digits).
* 3D (cc_mhd3d_main, M3:1132-1338), run to the third stored time: names,
  /x /y /z bit for bit, shapes (Nt, Nz, Ny, Nx), /t[0] within 1e-13, the
  first frame (stored after one step) of every field within 1e-12 of the
  reference's by its sum and maximum (the hybrid EOS's pow runs on the
  device; div B, roundoff itself, relative to |B| / dx)."""
from __future__ import annotations

import hashlib
import json
import subprocess
from pathlib import Path

import numpy as np
import pytest

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


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def _run(exe, *args):
    r = subprocess.run([str(ROOT / "core_collapse_b200" / exe), *map(str, args)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr


def test_mhd2d_driver_output_pinned_to_reference_main(tmp_path):
    fx = _fixture("mhd2d")
    out = tmp_path / "out"
    _run("cc_mhd2d_main", "--t_end", 0.02, "--out", out)
    names = [k.lstrip("/") for k in fx]
    assert sorted(p.stem for p in out.glob("*.npy")) == sorted(names)
    got = {k: np.load(out / f"{k}.npy") for k in names}
    for k in ("x", "y"):
        assert np.array_equal(got[k], _values(fx["/" + k]))
    t_ref = _values(fx["/t"])
    nt = len(got["t"])
    assert nt >= 3
    assert got["t"][0] == t_ref[0] and got["t"][1] == t_ref[1]
    assert np.allclose(got["t"], t_ref[:nt], rtol=1e-9, atol=0)
    for k in names[3:]:
        ent = fx["/" + k]
        assert list(got[k].shape) == [nt] + ent["dims"][1:], k
        assert _digest(got[k][0]) == ent["frames"][0]["sha256"], f"{k} t = 0 frame"


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
