"""The drop-in drivers' initial conditions and snapshots, pinned to the
reference's own main() (tests/golden/make_golden.py runs the compiled
reference once; see there).

* 2D (mhd2d_resistive_hlld_ct_gravity.cpp main(), M2:929-1139): with its
  default parameters the reference's core collapses near t = 0.275 and dt falls
  by orders of magnitude, so its main() never reaches t_end nor its HDF5 write
  in hours of CPU.  tests/golden/main_mhd2d_log.json keeps what it printed:
  max |div B| of the initial state and, per stored snapshot, t, dt (7
  significant digits) and max |div B| (12).  Here the library's host IC of that
  main (cc_ic_mhd2d_reference, M2:957-1048) with the reference's default
  Params, advanced by the oracle's restatement of the main loop with the
  reference's lexicographic SOR, prints the same strings for the first
  snapshots; the writer's dataset list is the one the driver mirrors.
* 3D (mhd3d_resistive_hlld_ct.cpp main(), M3:1132-1338): the library's host IC
  (cc_ic_mhd3d_reference, M3:1159-1272), one step of the oracle's main loop
  and its store (M3:1296-1321) equal the reference's first frame (stored after
  the first step) of all eleven fields bit for bit (SHA-256 of the FP64
  values, tests/golden/main_mhd3d.json: its HDF5 datasets, recorded in
  memory); /t[0] bit for bit; the dataset names, ranks and (Nt, Nz, Ny, Nx)
  shapes, which the driver's .npy output mirrors (checked on the GPU in
  test_gpu_main_pin.py)."""
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


def log_fixture() -> dict:
    f = GOLDEN / "main_mhd2d_log.json"
    if not f.exists():
        pytest.skip(f"{f.name} not generated (python tests/golden/make_golden.py --main2d-log-only)")
    return json.loads(f.read_text())


def test_mhd2d_main_log_and_writer_layout():
    fx = log_fixture()
    assert not fx["finished"] and len(fx["lines"]) >= 200
    ts = [float(ln[0]) for ln in fx["lines"]]
    assert all(b > a for a, b in zip(ts, ts[1:])) and 0.2 < ts[-1] < Params().t_end
    assert fx["datasets"] == [["/x", 1], ["/y", 1], ["/t", 1]] + [[f"/{k}", 3] for k in M2_FIELDS]


N_SNAPSHOTS = 6


def test_mhd2d_main_ic_and_first_snapshots_pinned():
    fx = log_fixture()
    p = Params()   # the reference's Params defaults (M2:44-86)
    U, B = ic_reference(p)
    cp = p.to_c()
    S = O.state_list(U, B)
    lib = O.oracle()
    assert f"{lib.or_mhd2d_divB_max(C.byref(cp), O.pp(S)):.12g}" == fx["init_max_divB"]
    t, next_store, got = 0.0, p.dt_store, []
    while len(got) < N_SNAPSHOTS:
        dt = lib.or_mhd2d_compute_dt(C.byref(cp), O.pp(S))
        S, t = O.m2_main_loop_oracle(cp, S, 1, mode=0, t0=t)   # mode 0: the reference's lexicographic SOR
        if t >= next_store - 1e-15:
            got.append([f"{t:.7g}", f"{dt:.7g}", f"{lib.or_mhd2d_divB_max(C.byref(cp), O.pp(S)):.12g}"])
            next_store += p.dt_store
    assert got == fx["lines"][:N_SNAPSHOTS]


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
