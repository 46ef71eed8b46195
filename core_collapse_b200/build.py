"""Build libcc_b200.so in-tree with nvcc for sm_100a.

    python -m core_collapse_b200.build [-v]

Translation units and their floating-point contract:
  mhd2d_f64.cu, mhd3d_f64.cu, euler2d_f64.cu,
  ns2d_f64.cu, common_kernels.cu, batch_f64.cu,
  batch_common.cu, noalloc.cu        -fmad=false: FP64 kernels round exactly like
                                     the reference's x86-64 build (no FMA)
  dpoisson.cu                        -fmad=false, explicit fma() only: the batched
                                     direct Poisson solve, reproducible on the CPU
  capi_adjoint.cu                    -fmad=false: the FP64 adjoint's kernels recompute
                                     FP64 forward intermediates and must round like them
  ic3d.cu                            -fmad=false: host IC of the 3D driver through the
                                     solver's EOS functions
  mhd2d_f32.cu, mhd3d_f32.cu, ns2d_f32.cu,
  euler2d_f32.cu, batch_f32.cu,
  adjoint_f32.cu                     FMA contraction on, approximate FP32 division
                                     and square root, flush-to-zero (the FP32 bulk path)
  capi*.cu, ic.cpp                   host code
and the host programs of MAINS (g++, linked against the library):
  main_mhd2d.cpp -> cc_mhd2d_main    drop-in for the reference's 2D MHD driver
  main_euler2d.cpp -> cc_euler2d_main  drop-in for the Euler/HLLC driver
  main_mhd3d.cpp -> cc_mhd3d_main    drop-in for the 3D MHD driver
  main_ns2d.cpp -> cc_ns2d_main      drop-in for the Navier-Stokes driver
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libcc_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", str(INCLUDE)]

UNITS = [
    ("mhd2d_f64.cu", ["-fmad=false"]),
    ("mhd3d_f64.cu", ["-fmad=false"]),
    ("euler2d_f64.cu", ["-fmad=false"]),
    ("ns2d_f64.cu", ["-fmad=false"]),
    ("common_kernels.cu", ["-fmad=false"]),
    ("noalloc.cu", ["-fmad=false"]),
    ("batch_f64.cu", ["-fmad=false"]),
    ("batch_common.cu", ["-fmad=false"]),
    ("dpoisson.cu", ["-fmad=false"]),
    ("capi_adjoint.cu", ["-fmad=false"]),
    ("ic3d.cu", ["-fmad=false"]),
    # FP32 bulk path: approximate division/sqrt (<= 2 ulp), denormals flushed
    ("mhd2d_f32.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("mhd3d_f32.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("euler2d_f32.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("ns2d_f32.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("batch_f32.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("adjoint_f32.cu", ["-prec-div=false", "-prec-sqrt=false", "-ftz=true"]),
    ("capi.cu", []),
    ("capi_mhd3d.cu", []),
    ("capi_euler2d.cu", []),
    ("capi_ns2d.cu", []),
    ("capi_batch.cu", []),
    ("ic.cpp", []),
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps(src: Path) -> list[Path]:
    return [src] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in _deps(src))


def build(verbose: bool = False, force: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    nv = nvcc()
    jobs = []
    for name, flags in UNITS:
        src = CSRC / name
        obj = BUILD / (name + ".o")
        cmd = [nv, *ARCH, *COMMON, *flags, "-c", str(src), "-o", str(obj)]
        if name.endswith(".cpp"):
            cmd = [nv, *COMMON, "-x", "c++", "-c", str(src), "-o", str(obj)]
        if verbose and name.endswith(".cu"):
            cmd.insert(1, "-Xptxas=-v")
        jobs.append((obj, src, cmd))
    todo = [(o, s, c) for o, s, c in jobs if force or _stale(o, s)]

    def run(job):
        obj, src, cmd = job
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
        return src.name, r.stderr

    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(todo)))) as ex:
        for name, err in ex.map(run, todo):
            if verbose and err:
                print(f"--- {name}\n{err}", file=sys.stderr)
    objs = [str(o) for o, _, _ in jobs]
    if todo or not LIB.exists() or any(Path(o).stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nv, *ARCH, "-shared", "-o", str(LIB), *objs, "-lcudart_static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_mains(verbose)
    return LIB


# host programs linked against the library (rpath $ORIGIN: they sit beside it)
MAINS = [("main_mhd2d.cpp", "cc_mhd2d_main"), ("main_euler2d.cpp", "cc_euler2d_main"),
         ("main_mhd3d.cpp", "cc_mhd3d_main"), ("main_ns2d.cpp", "cc_ns2d_main")]


def build_mains(verbose: bool = False) -> list[Path]:
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        raise RuntimeError("g++ not found (needed for the drop-in main programs)")
    outs = []
    for src_name, exe_name in MAINS:
        src, exe = CSRC / src_name, PKG / exe_name
        if not exe.exists() or exe.stat().st_mtime < max(LIB.stat().st_mtime, *(d.stat().st_mtime for d in _deps(src))):
            cmd = [cxx, "-O2", "-std=c++17", "-I", str(INCLUDE), str(src), "-L", str(PKG), "-lcc_b200",
                   "-Wl,-rpath,$ORIGIN", "-o", str(exe)]
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"building {exe_name} failed:\n{r.stdout}\n{r.stderr}")
            if verbose and r.stderr:
                print(r.stderr, file=sys.stderr)
        outs.append(exe)
    return outs


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
