"""Generate the golden fixtures of tests/golden/ from the compiled reference.

The reference solvers (mhd2d_resistive_hlld_ct_gravity.cpp,
mhd3d_resistive_hlld_ct.cpp, euler2d_gravity_hllc.cpp and the FFT Poisson of
navier_stokes_2d_hllc_poisson.cpp) are compiled in place into oracle/_ref/ by
oracle/Makefile.  This script runs them on the seeded cases of
tests/cases_*.py and stores inputs and reference outputs as .npz files, so
that tests/test_golden.py can pin the CPU oracle to the reference on a
machine without the reference tree.  Every stored output is the reference's
own result; nothing here is computed by the oracle or the library.

    python tests/golden/make_golden.py [--mains-only | --no-mains | --main2d-log-only]
    (from the repository root)

main_mhd3d.json holds what the reference's own 3D main() wrote (its HDF5
datasets, recorded in memory): dataset names and dimensions, the rank-1
datasets (x, y, z, t) in full, and of every field the SHA-256 digest and sum
of its first two stored frames and its last one.  The 2D main() does not
reach its HDF5 write with its default parameters (its core collapses and dt
falls by orders of magnitude near t = 0.275): main_mhd2d_log.json holds the
lines it printed per stored snapshot until it was stopped, and the dataset
list of its writer.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path[:0] = [str(HERE.parent.parent), str(HERE.parent)]

import oracle_lib as O  # noqa: E402
from cases_euler2d import CASES_EH, make_case_eh  # noqa: E402
from cases_mhd2d import CASES, make_case  # noqa: E402
from cases_mhd3d import CASES3, make_case3  # noqa: E402

MAIN_LOOP_STEPS = 3


def _params_json(kind: str, p) -> np.ndarray:
    return np.array(json.dumps({"kind": kind, "fields": dataclasses.asdict(p)}))


def _save(name: str, **arrays):
    np.savez_compressed(HERE / f"{name}.npz", **arrays)


def _state(prefix: str, S) -> dict:
    return {f"{prefix}{k}": np.asarray(a).copy() for k, a in enumerate(S)}


def mhd2d():
    R = O.ref("mhd2d")
    for name in sorted(CASES):
        p, U, B = make_case(name)
        cp = p.to_c()
        S = O.state_list(U, B)
        n = p.Nx * p.Ny
        gx, gy = np.zeros(n), np.zeros(n)
        if p.gravity_on:
            R.ref_mhd2d_poisson(C.byref(cp), O.dp(S[0]), O.dp(gx), O.dp(gy))
        dt = R.ref_mhd2d_compute_dt(C.byref(cp), O.pp(S))
        stage = O.m2_stage_ref(cp, S, gx, gy, dt)
        step = O.m2_rk2_ref(cp, S, gx, gy, dt)
        loop = O.copy_state(S)
        cp.t_end = 10.0
        t = C.c_double(0.0)
        R.ref_mhd2d_main_loop(C.byref(cp), O.pp(loop), MAIN_LOOP_STEPS, C.byref(t))
        divb = R.ref_mhd2d_divB_max(C.byref(cp), O.pp(loop))
        _save(f"mhd2d_{name}", params=_params_json("mhd2d", p), gx=gx, gy=gy, dt=np.float64(dt),
              loop_t=np.float64(t.value), loop_divb=np.float64(divb),
              **_state("in", S), **_state("stage", stage), **_state("step", step), **_state("loop", loop))


def mhd3d():
    R = O.ref("mhd3d")
    for name in sorted(CASES3):
        p, s = make_case3(name)
        cp = p.to_c()
        S = [a.copy() for a in s.arrays()]
        dt = R.ref_mhd3d_compute_dt(C.byref(cp), O.pp(S))
        stage = O.copy_state(S)
        R.ref_mhd3d_advance_stage(C.byref(cp), O.pp(S), O.pp(stage), dt)
        step = O.m3_rk2_ref(cp, S, dt)
        loop = O.copy_state(S)
        cp.t_end = 10.0
        t = C.c_double(0.0)
        R.ref_mhd3d_main_loop(C.byref(cp), O.pp(loop), MAIN_LOOP_STEPS, C.byref(t))
        divb = R.ref_mhd3d_divB_max(C.byref(cp), O.pp(loop))
        _save(f"mhd3d_{name}", params=_params_json("mhd3d", p), dt=np.float64(dt), loop_t=np.float64(t.value),
              loop_divb=np.float64(divb),
              **_state("in", S), **_state("stage", stage), **_state("step", step), **_state("loop", loop))


def euler2d():
    from core_collapse_b200.euler2d import ParamsEH
    R = O.ref("euler2d")
    for name in sorted(CASES_EH):
        p, s = make_case_eh(name)   # the reference's SOR is fixed at omega 1.7, tol 1e-10 (EH:328-330)
        cp = p.to_c()
        S = [a.copy() for a in s.arrays()]
        dt = R.ref_euler2d_compute_dt(C.byref(cp), O.pp(S))
        rhs = [np.zeros_like(a) for a in S]
        R.ref_euler2d_rhs(C.byref(cp), O.pp(S), O.pp(rhs))
        step = O.copy_state(S)
        R.ref_euler2d_rk2_step(C.byref(cp), O.pp(step), dt)
        _save(f"euler2d_{name}", params=_params_json("euler2d", p), dt=np.float64(dt),
              **_state("in", S), **_state("rhs", rhs), **_state("step", step))
    # the reference's own main(): random-blob IC, tolerance SOR, 3 steps
    p = ParamsEH(Nx=16, Ny=12)
    cp = p.to_c()
    n = p.Nx * p.Ny
    S = [np.zeros(n) for _ in range(4)]
    R.ref_euler2d_init_random_blob(C.byref(cp), O.pp(S))
    loop = O.copy_state(S)
    t = C.c_double(0.0)
    rc = R.ref_euler2d_main_loop(C.byref(cp), O.pp(loop), MAIN_LOOP_STEPS, C.byref(t))
    assert rc == 0
    _save("euler2d_random_blob", params=_params_json("euler2d", p), loop_t=np.float64(t.value),
          **_state("ic", S), **_state("loop", loop))


def fft():
    R = O.ref("fft")
    rng = np.random.default_rng(11)
    out = {}
    for n in (8, 64):
        for inv in (0, 1):
            z = rng.normal(size=2 * n)
            a = z.copy()
            R.ref_fft1d(n, O.dp(a), inv)
            out[f"fft1d_{n}_{inv}_in"], out[f"fft1d_{n}_{inv}_out"] = z, a
    for nx, ny in ((16, 16), (32, 8)):
        rho = 1.0 + rng.random(nx * ny)
        phi = np.zeros(nx * ny)
        R.ref_fft_poisson(nx, ny, -1.0, 1.0, -1.0, 1.0, 1.0, O.dp(rho), O.dp(phi))
        out[f"poisson_{nx}x{ny}_rho"], out[f"poisson_{nx}x{ny}_phi"] = rho, phi
    _save("fft", **out)


def frame_digest(a: np.ndarray) -> str:
    """SHA-256 of a frame's FP64 values (little-endian bytes)."""
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<f8").tobytes()).hexdigest()


def read_record(path: Path) -> dict:
    """The datasets the reference's writer produced, as written by
    oracle/_ref/ref_main_record: name -> {file, dims, values (rank 1) or the
    SHA-256 digest, sum and max |value| of the first two frames and the last
    one (rank >= 2)}."""
    b = path.read_bytes()
    assert b[:8] == b"CCH5REC1"
    off = 8

    def take(nbytes, dtype, n):
        nonlocal off
        a = np.frombuffer(b, dtype=dtype, count=n, offset=off)
        off += nbytes * n
        return a

    out = {}
    n = int(take(4, "<i4", 1)[0])
    for _ in range(n):
        strs = []
        for _k in range(2):
            ln = int(take(4, "<i4", 1)[0])
            strs.append(b[off:off + ln].decode())
            off += ln
        rank = int(take(4, "<i4", 1)[0])
        dims = [int(d) for d in take(8, "<u8", rank)]
        head = take(8, "<f8", int(take(8, "<i8", 1)[0]))
        last = take(8, "<f8", int(take(8, "<i8", 1)[0]))
        ent = {"file": strs[1], "dims": dims}
        if rank == 1:
            ent["values"] = [float(v).hex() for v in head]
        else:
            frame = int(np.prod(dims[1:]))
            frames = [head[k * frame:(k + 1) * frame] for k in range(len(head) // frame)] + [last]
            ent["frames"] = [{"sha256": frame_digest(a), "sum": float(np.sum(a)), "absmax": float(np.max(np.abs(a)))}
                             for a in frames]
            ent["frame_index"] = list(range(len(frames) - 1)) + [dims[0] - 1]
        out[strs[0]] = ent
    return out


def write_main_fixture(name: str, record: Path):
    (HERE / f"main_{name}.json").write_text(json.dumps(read_record(record), indent=1) + "\n")


MAIN2D_SECONDS = 1200   # wall time allowed to the reference's 2D main() (see main2d_log)


def _writer_datasets(src: Path, writer: str) -> list[list]:
    """[name, rank] of every dataset the reference's HDF5 writer `writer`
    writes, in order, read from its source (write1 -> rank 1, write3 -> rank 3)."""
    import re
    text = src.read_text()
    body = text[text.index(f"static void {writer}("):]
    body = body[:body.index("H5Fclose(file);")]
    return [[name, 1 if kind == "1" else 3] for kind, name in re.findall(r'write([13])\("(/\w+)"', body)]


def main2d_log(seconds: int = MAIN2D_SECONDS):
    """The reference's own 2D main() (mhd2d_resistive_hlld_ct_gravity.cpp
    main(), M2:929-1139) with its default parameters, run in a plain process
    (oracle/_ref/ref_main_record): every line it prints, one per stored
    snapshot ("t=... dt=... max|divB|=...", M2:1119-1125, t and dt to 7
    significant digits, div B to 12).  With its defaults the core collapses
    near t = 0.275 and dt falls by orders of magnitude, so the run does not
    reach t_end = 0.35 (nor its HDF5 write) in hours; it is stopped after
    `seconds` of wall time and the lines printed so far are kept, with the
    dataset list of its writer (write_h5, M2:881-925) read from the source."""
    import subprocess
    import tempfile
    import threading
    import time
    runner = O.REF_DIR / "ref_main_record"
    lines, init = [], None
    t0 = time.time()
    with tempfile.TemporaryDirectory() as tmp:
        proc = subprocess.Popen([str(runner), str(O.REF_DIR / "libref_mhd2d.so"), "ref_mhd2d_run_main",
                                 str(Path(tmp) / "rec.bin")], cwd=tmp, stdout=subprocess.PIPE, text=True, bufsize=1)
        timer = threading.Timer(seconds, proc.kill)
        timer.start()
        try:
            for ln in proc.stdout:
                ln = ln.strip()
                if ln.startswith("init max|divB|="):
                    init = ln.split("=", 1)[1]
                elif ln.startswith("t="):
                    kv = dict(part.split("=", 1) for part in ln.split())
                    lines.append([kv["t"], kv["dt"], kv["max|divB|"], round(time.time() - t0, 1)])
        finally:
            timer.cancel()
            proc.wait()
    fx = {
        "source": "mhd2d_resistive_hlld_ct_gravity.cpp main() with its default Params, stdout",
        "finished": proc.returncode == 0,
        "wall_seconds_allowed": seconds,
        "seconds_to_last_line": lines[-1][3] if lines else None,
        "init_max_divB": init,
        "columns": ["t", "dt", "max|divB|"],
        "lines": [ln[:3] for ln in lines],
        "datasets": _writer_datasets(O.REFERENCE_SRC / "mhd2d_resistive_hlld_ct_gravity.cpp", "write_h5"),
    }
    (HERE / "main_mhd2d_log.json").write_text(json.dumps(fx, indent=0) + "\n")


def mains():
    """The reference's own main() of the 3D MHD solver, run once with its
    defaults in a plain process (oracle/_ref/ref_main_record): its HDF5
    datasets, recorded in memory by oracle/hdf5_stub/hdf5.h, go to
    main_mhd3d.json.  The 2D main() does not finish with its defaults (see
    main2d_log): its printed lines go to main_mhd2d_log.json."""
    import subprocess
    import tempfile
    runner = O.REF_DIR / "ref_main_record"
    for name in ("mhd3d",):
        with tempfile.TemporaryDirectory() as tmp:
            rec = Path(tmp) / "rec.bin"
            subprocess.run([str(runner), str(O.REF_DIR / f"libref_{name}.so"), f"ref_{name}_run_main", str(rec)],
                           check=True, stdout=subprocess.DEVNULL, cwd=tmp)
            write_main_fixture(name, rec)
    main2d_log()


def main():
    for name in ("mhd2d", "mhd3d", "euler2d", "fft"):
        if O.ref(name) is None:
            raise SystemExit(f"compiled reference libref_{name}.so is missing: run make -C oracle")
    if "--main2d-log-only" in sys.argv:
        main2d_log()
        return
    if "--mains-only" not in sys.argv:
        mhd2d()
        mhd3d()
        euler2d()
        fft()
    if "--no-mains" not in sys.argv:
        mains()
    print("wrote", sorted(p.name for p in HERE.glob("*.npz")) + sorted(p.name for p in HERE.glob("main_*.json")))


if __name__ == "__main__":
    main()
