"""Build the host-only test harnesses of tests/native/ (nvcc, no GPU needed)."""
from __future__ import annotations

import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = HERE / "_build"


def build(name: str = "adj_local") -> Path:
    src = HERE / f"{name}.cu"
    lib = OUT / f"lib{name}.so"
    deps = [src] + list((ROOT / "core_collapse_b200" / "csrc").glob("*.cuh"))
    if lib.exists() and all(lib.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return lib
    OUT.mkdir(exist_ok=True)
    cmd = ["nvcc", "-O2", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-fmad=false",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-I", str(ROOT / "core_collapse_b200" / "csrc"), "-I", str(ROOT / "include"), str(src), "-o", str(lib)]
    subprocess.run(cmd, check=True)
    return lib
