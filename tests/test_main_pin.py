"""The drop-in drivers' initial conditions and snapshot fields, pinned to
what the reference's own main() wrote (tests/golden/main_mhd2d.json and
main_mhd3d.json: its HDF5 datasets, recorded by running the compiled
reference once with a recording hdf5.h; see tests/golden/make_golden.py).

* 2D (mhd2d_resistive_hlld_ct_gravity.cpp main(), M2:929-1139): the library's
  host IC of that main (cc_ic_mhd2d_reference, M2:957-1048) with the
  reference's default Params, turned into the ten snapshot fields by the
  oracle's restatement of the store (M2:1065-1106), equals the reference's
  t = 0 frame of /rho /P /Mach /u /v /vabs /Bx /By /Bz /divB bit for bit
  (SHA-256 of the FP64 values); /x and /y bit for bit; /t[0] = 0.
* 3D (mhd3d_resistive_hlld_ct.cpp main(), M3:1132-1338): the library's host IC
  (cc_ic_mhd3d_reference, M3:1159-1272), one step of the oracle's main loop
  and its store (M3:1296-1321) equal the reference's first frame (stored after
  the first step) of all eleven fields bit for bit; /t[0] bit for bit.
* The dataset layout: names, ranks and (Nt, [Nz,] Ny, Nx) shapes, which the
  drivers' .npy output mirrors (checked on the GPU in test_gpu_main_pin.py)."""
import ctypes as C
import hashlib
import json
from pathlib import Path

import numpy as np
import pytest

import oracle_lib as O
from core_collapse_b200.mhd2d import Params, ic_reference
from core_collapse_b200.mhd3d import Params3, ic_reference3

GOLDEN = Path(__file__).resolve().parent / "golden"
M2_FIELDS = ["rho", "P", "Mach", "u", "v", "vabs", "Bx", "By", "Bz", "divB"]
M3_FIELDS = ["rho", "P", "Mach", "u", "v", "w", "vabs", "Bx", "By", "Bz", "divB"]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def fixture(name: str) -> dict:
    f = GOLDEN / f"main_{name}.json"
    if not f.exists():
        pytest.skip(f"{f.name} not generated (python tests/golden/make_golden.py --mains-only)")
    return json.loads(f.read_text())


def values(ent) -> np.ndarray:
    return np.array([float.fromhex(v) for v in ent["values"]])


def test_mhd2d_main_layout():
    fx = fixture("mhd2d")
    p = Params()
    assert list(fx) == ["/x", "/y", "/t"] + [f"/{k}" for k in M2_FIELDS]
    nt = fx["/t"]["dims"][0]
    assert fx["/x"]["dims"] == [p.Nx] and fx["/y"]["dims"] == [p.Ny]
    for k in M2_FIELDS:
        assert fx[f"/{k}"]["dims"] == [nt, p.Ny, p.Nx]
        assert fx[f"/{k}"]["file"] == "out2d_mhd.h5"


def test_mhd2d_main_ic_and_store_pinned():
    fx = fixture("mhd2d")
    p = Params()   # the reference's Params defaults (M2:44-86)
    U, B = ic_reference(p)
    derived = O.m2_derived_oracle(p.to_c(), O.state_list(U, B))
    dx, dy = (p.x1 - p.x0) / p.Nx, (p.y1 - p.y0) / p.Ny
    assert np.array_equal(values(fx["/x"]), p.x0 + (np.arange(p.Nx) + 0.5) * dx)
    assert np.array_equal(values(fx["/y"]), p.y0 + (np.arange(p.Ny) + 0.5) * dy)
    assert values(fx["/t"])[0] == 0.0
    for k, a in zip(M2_FIELDS, derived):
        assert digest(a) == fx[f"/{k}"]["frames"][0]["sha256"], f"/{k} frame 0"


def test_mhd3d_main_layout():
    fx = fixture("mhd3d")
    p = Params3()
    assert list(fx) == ["/x", "/y", "/z", "/t"] + [f"/{k}" for k in M3_FIELDS]
    nt = fx["/t"]["dims"][0]
    for k in M3_FIELDS:
        assert fx[f"/{k}"]["dims"] == [nt, p.Nz, p.Ny, p.Nx]
        assert fx[f"/{k}"]["file"] == "out3d_mhd.h5"


def test_mhd3d_main_first_frame_pinned():
    fx = fixture("mhd3d")
    p = Params3()  # the reference's Params defaults (M3:43-89)
    s = ic_reference3(p)
    cp = p.to_c()
    S, t = O.m3_main_loop_oracle(cp, [a.copy() for a in s.arrays()], 1)
    assert t == values(fx["/t"])[0]
    for ax, n0, lo, hi in (("/x", p.Nx, p.x0, p.x1), ("/y", p.Ny, p.y0, p.y1), ("/z", p.Nz, p.z0, p.z1)):
        assert np.array_equal(values(fx[ax]), lo + (np.arange(n0) + 0.5) * ((hi - lo) / n0))
    n = p.Nx * p.Ny * p.Nz
    out = [np.empty(n) for _ in M3_FIELDS]
    O.oracle().or_mhd3d_derived(C.byref(cp), O.pp(S), O.pp(out))
    for k, a in zip(M3_FIELDS, out):
        assert digest(a) == fx[f"/{k}"]["frames"][0]["sha256"], f"/{k} frame 0"
