#!/usr/bin/env python
"""Benchmark of the 2D resistive-MHD + self-gravity step (the FFT-gravity
precision-ladder workload: 4096^2 periodic [-1,1]^2, Orszag-Tang fields plus a
Gaussian density core of amplitude 4 and width 0.1, gamma 5/3, G 1,
eta 1e-3, CFL 0.4).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line on stdout (rank 0).  `value` is FP32 zone-updates/s over all
ranks (weak scaling: each rank advances its own instance), with the FP64 path
timed on the same workload beside it and the FP32-vs-FP64 L1 error stated.
A step is one pass of the reference's main-loop body: Poisson(rho), dt,
rk2_step (two stages with a second Poisson solve between them).

--impl reference times the CPU implementation of the same path (the oracle
port of the reference step and its spectral Poisson solve, FP64, one
independent instance per host thread) on rank 0 and prints the same line with
"impl": "reference"."""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

METRIC = "zone-updates/s FP32 vs FP64 on GPU at stated L1 err; adjoint/forward time ratio"
UNIT = "zone-updates/s"
# algorithmic FP words per cell of one stage-kernel launch: state in (6 cell + 2
# face), the potential, state out (6 cell + 2 face)
STAGE_WORDS = 17
# algorithmic FP words per zone-update of a whole RK2 step with gravity
STEP_WORDS = 42


def workload_params(n: int, precision: str):
    from core_collapse_b200.mhd2d import Params
    return Params(Nx=n, Ny=n, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=True, periodic_y=True, gamma=5.0 / 3.0,
                  G=1.0, eta=1e-3, cfl=0.4, gravity_on=True, poisson="fft", precision=precision, t_end=1e30)


def measured_peaks() -> dict:
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


# ---------------------------------------------------------------- CPU baseline

def cpu_threads() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except Exception:
        return max(1, os.cpu_count() or 1)


def cpu_run(sample_n: int, nthreads: int, nsteps: int) -> tuple[float, float]:
    """Advance `nthreads` independent sample_n^2 instances by nsteps each, one
    per thread, with the CPU port of the reference step (FP64, spectral
    gravity).  Returns (wall seconds, zone-updates)."""
    import ctypes as C

    import oracle_lib as O
    p = workload_params(sample_n, "fp64")
    S0 = ic_orszag_tang_numpy(p, core_amp=4.0, core_width=0.1)
    cp = p.to_c()
    states = [[a.copy() for a in S0] for _ in range(nthreads)]
    ptrs = [O.pp(s) for s in states]
    orc = O.oracle()

    def work(k):
        t = C.c_double(0.0)
        orc.or_mhd2d_main_loop(C.byref(cp), ptrs[k], nsteps, C.byref(t), 2, 0)

    th = [threading.Thread(target=work, args=(k,)) for k in range(nthreads)]
    t0 = time.perf_counter()
    for t in th:
        t.start()
    for t in th:
        t.join()
    wall = time.perf_counter() - t0
    return wall, float(nthreads) * sample_n * sample_n * nsteps


def ic_orszag_tang_numpy(p, core_amp: float, core_width: float) -> list:
    """The benchmark's initial state in the reference layouts, built with numpy
    so that the CPU legs never load the GPU library: Orszag-Tang fields, face B
    from the corner potential Az = B0 (cos(2 pi y) / (2 pi) + cos(4 pi x) / (4 pi)),
    B0 = 1/sqrt(4 pi), rho = 25/(36 pi) + a Gaussian core, P = 5/(12 pi),
    conserved through the reference's prim_to_cons (M2:137-146) with B at cell
    centres from the face averages.  Returns [rho, mx, my, mz, E, Bz, Bx_f, By_f]."""
    import numpy as np
    nx, ny = p.Nx, p.Ny
    dx, dy = (p.x1 - p.x0) / nx, (p.y1 - p.y0) / ny
    B0 = 1.0 / np.sqrt(4.0 * np.pi)
    X = p.x0 + np.arange(nx + 1) * dx
    Y = p.y0 + np.arange(ny + 1) * dy
    Az = B0 * (np.cos(2.0 * np.pi * Y)[:, None] / (2.0 * np.pi) + np.cos(4.0 * np.pi * X)[None, :] / (4.0 * np.pi))
    bx = (Az[1:, :] - Az[:-1, :]) / dy            # (ny, nx+1)
    by = -(Az[:, 1:] - Az[:, :-1]) / dx           # (ny+1, nx)
    xc = p.x0 + (np.arange(nx) + 0.5) * dx
    yc = p.y0 + (np.arange(ny) + 0.5) * dy
    cx, cy = 0.5 * (p.x0 + p.x1), 0.5 * (p.y0 + p.y1)
    r2 = (xc[None, :] - cx) ** 2 + (yc[:, None] - cy) ** 2
    rho = np.maximum(25.0 / (36.0 * np.pi) + core_amp * np.exp(-r2 / (2.0 * core_width ** 2)), p.floor_rho)
    u = np.broadcast_to(-np.sin(2.0 * np.pi * yc)[:, None], (ny, nx))
    v = np.broadcast_to(np.sin(2.0 * np.pi * xc)[None, :], (ny, nx))
    P = np.full((ny, nx), max(5.0 / (12.0 * np.pi), p.floor_P))
    Bxc = 0.5 * (bx[:, :-1] + bx[:, 1:])
    Byc = 0.5 * (by[:-1, :] + by[1:, :])
    E = P / (p.gamma - 1.0) + 0.5 * rho * (u * u + v * v) + 0.5 * (Bxc * Bxc + Byc * Byc)
    z = np.zeros(nx * ny)
    return [np.ascontiguousarray(a).ravel() for a in (rho, rho * u, rho * v)] + [z.copy(), E.ravel().copy(), z.copy(),
                                                                                  bx.ravel().copy(), by.ravel().copy()]


def cpu_baseline(sample_n: int, nsteps: int) -> dict:
    n = cpu_threads()
    wall, zu = cpu_run(sample_n, n, nsteps)
    return {"value": zu / wall, "unit": UNIT, "cores": n, "kind": "port",
            "sample": f"{nsteps} step(s) of an independent {sample_n}^2 instance of the same workload per thread, "
                      f"{n} threads, FP64 oracle port (bitwise-pinned to the reference step and spectral solve), "
                      f"{wall:.1f} s wall"}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = cpu_threads()
    sample_n = args.cpu_sample_grid
    for _ in range(args.warmup):
        cpu_run(sample_n, n, 1)
    walls = []
    zus = 0.0
    for _ in range(args.steps):
        w, zu = cpu_run(sample_n, n, 1)
        walls.append(w)
        zus += zu
    total = sum(walls)
    value = zus / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_block(args),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": n, "kind": "port",
                         "sample": f"each step: one RK2 step of an independent {sample_n}^2 instance of the workload "
                                   f"per thread on {n} threads (FP64 CPU port of the reference step + spectral "
                                   f"Poisson; the reference's own M2 step has no spectral solve)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_block(args) -> dict:
    return {"workload": f"2D resistive MHD HLLD+CT + FFT self-gravity, {args.grid}^2 periodic [-1,1]^2, "
                        f"Orszag-Tang + Gaussian core (amp 4, width 0.1), gamma 5/3, G 1, eta 1e-3, CFL 0.4",
            "grid": [args.grid, args.grid], "cells_per_gpu": args.grid * args.grid,
            "poisson": "fft (2 solves per step)", "precision_headline": "fp32 bulk, fp64 reductions",
            "l2_policy": "inputs larger than L2 (state buffer >= 537 MB at 4096^2 FP32)",
            "parallelism": f"{args.gpus} independent instance(s), one per GPU"}


# ---------------------------------------------------------------- clocks

class ClockSampler:
    """NVML samples of the SM clock and throttle reasons during a region."""

    def __init__(self, device_index: int, period_s: float = 0.02):
        self.idx = device_index
        self.period = period_s
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = threading.Event()
        self._th = None
        self.ok = False

    def __enter__(self):
        try:
            import pynvml as N
            N.nvmlInit()
            self._N = N
            self._h = N.nvmlDeviceGetHandleByIndex(self.idx)
            self.max_mhz = N.nvmlDeviceGetMaxClockInfo(self._h, N.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False
            return self
        names = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
                 "sw_power_cap": 0x4, "hw_power_brake_slowdown": 0x80}

        def loop():
            N = self._N
            while not self._stop.is_set():
                try:
                    self.samples.append(N.nvmlDeviceGetClockInfo(self._h, N.NVML_CLOCK_SM))
                    r = N.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                    for k, bit in names.items():
                        if r & bit:
                            self.reasons.add(k)
                except Exception:
                    pass
                time.sleep(self.period)

        self._th = threading.Thread(target=loop, daemon=True)
        self._th.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._th:
            self._th.join()

    def summary(self) -> dict:
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": 0}
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ---------------------------------------------------------------- GPU arm

def stage_capture(grid: int, key: str):
    """A per-launch figure of the stage kernel (DRAM bytes, warp instructions)
    from the committed ncu capture, scaled to the benchmark grid by cell count
    (both grow with the cells: every tile reads its halo once and runs the same
    work per cell)."""
    f = ROOT / "profiles" / "stage_kernel_traffic.json"
    if not f.exists():
        return None
    d = json.loads(f.read_text())
    try:
        return float(d[key]) * (grid * grid) / float(d["cells"])
    except Exception:
        return None


def traffic_per_launch(grid: int):
    return stage_capture(grid, "dram_bytes_per_launch")


def issue_roofline(grid: int, launch_ms: float, clk) -> dict | None:
    """The stage kernel's instruction-issue bound: its warp instructions per
    launch (ncu capture, scaled to the grid) over 148 SMs x 4 schedulers x one
    instruction per cycle at the SM clock sampled during the timed region."""
    inst = stage_capture(grid, "warp_instructions_per_launch")
    mhz = (clk or {}).get("sm_mhz") or (clk or {}).get("sm_max_mhz") or 1965
    if not inst or not launch_ms:
        return None
    ms = inst / (148 * 4 * mhz * 1e6) * 1e3
    return {"warp_instructions_per_launch": inst, "sm_mhz": mhz, "bound_ms": ms, "frac": ms / launch_ms}


def run_ours(args) -> None:
    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    from core_collapse_b200.mhd2d import Mhd2dSolver, ic_orszag_tang

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    n = args.grid
    cells = n * n
    # a non-default stream shared by the library and the timing events (the
    # legacy null stream has handle 0, which the C ABI reads as "own stream")
    stream = torch.cuda.Stream()
    p32 = workload_params(n, "fp32")
    U0, B0 = ic_orszag_tang(p32, core_amp=4.0, core_width=0.1)

    def timed_run(precision: str, profile: bool, clocks: bool):
        p = workload_params(n, precision)
        s = Mhd2dSolver(p)
        s.set_stream(stream.cuda_stream)
        if precision == "fp32":
            s.set_stage_kernel(args.stage_kernel, args.march_rows)
        s.upload(U0, B0)
        s.advance(args.warmup, 0.0)
        s.set_profiling(profile)
        s.reset_perf()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local) if clocks else None
        if sampler:
            sampler.__enter__()
        e0.record(stream)
        s.advance(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        if sampler:
            sampler.__exit__()
        barrier()
        ms = e0.elapsed_time(e1)
        perf = s.perf()
        return s, ms, perf, (sampler.summary() if sampler else None)

    # FP32 headline
    s32, ms32, perf32, clk = timed_run("fp32", profile=True, clocks=True)
    ms32_max = max_over_ranks(ms32)
    value32 = world * cells * args.steps / (ms32_max / 1000.0)
    stage_avg_ms = perf32["stage_ms"] / max(1, perf32["stage_launches"])
    stage_bytes = STAGE_WORDS * 4 * cells

    # FP64 on the same workload and step count
    s64, ms64, perf64, _ = timed_run("fp64", profile=True, clocks=False)
    ms64_max = max_over_ranks(ms64)
    value64 = world * cells * args.steps / (ms64_max / 1000.0)
    stage64_avg_ms = perf64["stage_ms"] / max(1, perf64["stage_launches"])

    d32 = s32.diagnostics()

    # end to end through the C ABI with pinned host buffers, copies timed every
    # step: upload the state, one main-loop step, download the state
    pin = lambda m: torch.empty(m, dtype=torch.float64, pin_memory=True).numpy()
    from core_collapse_b200.mhd2d import Bfaces, Ucc
    Uh = Ucc(*[pin(cells) for _ in range(6)])
    Bh = Bfaces(pin((n + 1) * n), pin(n * (n + 1)))
    h2d = sum(a.nbytes for a in Uh.arrays()) + Bh.Bx_f.nbytes + Bh.By_f.nbytes
    e2e_steps = max(1, min(args.steps, args.e2e_steps))

    def e2e(s) -> float:
        for a, b in zip(Uh.arrays() + [Bh.Bx_f, Bh.By_f], U0.arrays() + [B0.Bx_f, B0.By_f]):
            a[:] = b
        s.set_profiling(False)
        s.reset_perf()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(e2e_steps):
            s.upload(Uh, Bh)
            s.advance(1)
            s.download(Uh, Bh)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return world * cells * e2e_steps / (max_over_ranks(e0.elapsed_time(e1)) / 1000.0)

    e2e_value = e2e(s32)
    e2e64_value = e2e(s64)
    s32.close()
    s64.close()

    peaks = measured_peaks()
    achieved = stage_bytes / (stage_avg_ms / 1000.0) / 1e9
    line = {
        "metric": METRIC, "value": value32, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms32_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config_block(args),
        "fp64": {"value": value64, "ms_per_step": ms64_max / args.steps, "dtype": "f64",
                 "stage_kernel_ms": stage64_avg_ms,
                 "stage_kernel_gbs": STAGE_WORDS * 8 * cells / (stage64_avg_ms / 1000.0) / 1e9,
                 "e2e": {"value": e2e64_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                         "steps": e2e_steps, "api": "cc_mhd2d_upload + cc_mhd2d_advance(1) + cc_mhd2d_download, "
                                                    "pinned FP64 host"}},
        "fp32_over_fp64": value32 / value64,
        "roofline": {"bound": "hbm", "kernel": ("m2_march_kernel<float>" if args.stage_kernel == "march"
                                                else "m2_stage_kernel<float>") + " (one RK2 stage)",
                     "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                     "traffic": traffic_per_launch(n), "algorithmic_bytes_per_launch": stage_bytes,
                     "launch_ms": stage_avg_ms,
                     "step_roofline_frac": STEP_WORDS * 4 * value32 / world / 1e9 / peaks["hbm_gbs"],
                     "issue": issue_roofline(n, stage_avg_ms, clk)},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                "steps": e2e_steps, "api": "cc_mhd2d_upload + cc_mhd2d_advance(1) + cc_mhd2d_download, pinned FP64 host"},
        "gpu_launches": perf32["kernel_launches"],
        "clocks": clk,
        "max_divB_fp32": d32["max_divB"],
    }
    if world == 1 and not args.skip_ladder:
        lad = run_ladder(args, stream)
        line["precision_ladder"] = lad
        big = lad["grids"][str(max(int(g) for g in lad["grids"]))]
        line["l1_err"] = big["fp32"]["l1_max"]
        line["linf_err"] = big["fp32"]["linf_max"]
    if world == 1 and not args.skip_3d:
        line["mhd3d"] = run_3d(args, stream)
    if world == 1 and not args.skip_ns:
        line["ns2d"] = run_ns2d(args, stream, peaks)
    if world == 1 and not args.skip_eh:
        line["euler2d"] = run_euler2d(args, stream, peaks)
    if not args.skip_ensemble:
        line["ensemble"] = run_ensemble(args, stream, rank, world, barrier, max_over_ranks, value32 / world)
    if world == 1 and not args.skip_adjoint:
        line["adjoint"] = run_adjoint(args, stream)
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_sample_grid, args.cpu_steps)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


STATE_FIELDS = ["rho", "mx", "my", "mz", "E", "Bz", "Bx_f", "By_f"]


def field_errors(got: list, want: list) -> dict:
    """Per-field relative errors of a state against a reference state:
    L1 = sum|a - b| / sum|b| and L-inf = max|a - b| / max|b| (absolute where
    the reference field is identically zero)."""
    import numpy as np
    l1, linf = {}, {}
    for name, a, b in zip(STATE_FIELDS, got, want):
        d = np.abs(a - b)
        s1, sm = float(np.sum(np.abs(b))), float(np.max(np.abs(b)))
        l1[name] = float(np.sum(d)) / s1 if s1 > 0 else float(np.max(d))
        linf[name] = float(np.max(d)) / sm if sm > 0 else float(np.max(d))
    return {"l1": l1, "linf": linf, "l1_max": max(l1.values()), "linf_max": max(linf.values())}


def run_ladder(args, stream) -> dict:
    """Precision ladder of the FFT-gravity workload: from the same initial
    state, FP64 runs --ladder-steps steps to t_final, then FP32 (plain, and
    with the compensated state update) runs to the same t_final (its own CFL
    steps, the last one clamped to t_final); each FP32 state is compared with
    the FP64 one per field (L1, L-inf).  The FP64 GPU path stands in for the
    oracle here: it matches the CPU restatement of the reference step to
    <= 1e-12 (tests/test_gpu_config_scale.py runs that comparison at 256^2
    and 1024^2)."""
    import torch

    from core_collapse_b200.mhd2d import Mhd2dSolver, ic_orszag_tang
    import oracle_lib as O
    out = {"steps": args.ladder_steps, "workload": "the benchmark workload at each grid, from t = 0",
           "reference": "GPU FP64 path (pinned to the CPU oracle at <= 1e-12 by the config-scale parity tests)",
           "grids": {}}
    for n in [int(g) for g in args.ladder_grids.split(",") if g]:
        p64 = workload_params(n, "fp64")
        U0, B0 = ic_orszag_tang(p64, core_amp=4.0, core_width=0.1)
        blk = {}

        def run(p, nsteps):
            with Mhd2dSolver(p) as s:
                s.set_stream(stream.cuda_stream)
                s.upload(U0, B0)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                t = s.advance(nsteps, 0.0)
                e1.record(stream)
                torch.cuda.synchronize()
                U, B = s.download()
                d = s.diagnostics()
            return O.state_list(U, B), t, e0.elapsed_time(e1), d

        S64, t64, ms64, d64 = run(p64, args.ladder_steps)
        blk["t_final"] = t64
        blk["fp64"] = {"ms": ms64, "steps": args.ladder_steps, "ms_per_step": ms64 / args.ladder_steps,
                       "max_divB": d64["max_divB"]}
        for tag, extra in (("fp32", {}), ("fp32_compensated", {"compensated": True})):
            p = workload_params(n, "fp32")
            p.t_end = t64
            for k, v in extra.items():
                setattr(p, k, v)
            S, t, ms, d = run(p, args.ladder_steps + args.ladder_steps // 10 + 2)
            e = field_errors(S, S64)
            e.update({"t_final": t, "steps": d["steps"], "ms": ms, "ms_per_step": ms / max(1, d["steps"]),
                      "max_divB": d["max_divB"]})
            blk[tag] = e
        out["grids"][str(n)] = blk
    return out


def run_3d(args, stream) -> dict:
    """3D resistive HLLD+CT workload: 256^3 periodic unit cube, ideal gas
    gamma 5/3 (hybrid EOS with K1 = Kbounce = 0), eta 5e-4, rho 1, p 1/gamma,
    random-phase v and A with 1 <= |k| <= 4 (seed 1), rms v 0.5, rms B 0.3."""
    import torch

    from core_collapse_b200.mhd3d import Mhd3dSolver, Params3, ic_turbulence3d
    n = args.grid3d
    steps = max(1, args.steps3d)
    s0 = ic_turbulence3d(Params3.ideal_gas(Nx=n, Ny=n, Nz=n), seed=1)
    out = {"workload": f"3D resistive MHD HLLD+CT, {n}^3 periodic, random-phase v and A (|k| in [1,4], seed 1), "
                       f"rms v 0.5, rms B 0.3, eta 5e-4, CFL 0.4", "steps": steps, "warmup": args.warmup}
    for prec in ("fp32", "fp64"):
        p = Params3.ideal_gas(Nx=n, Ny=n, Nz=n, eta=5e-4, cfl=0.4, precision=prec, t_end=1e30)
        with Mhd3dSolver(p) as g:
            g.set_stream(stream.cuda_stream)
            g.upload(s0)
            d0 = g.diagnostics()
            g.advance(args.warmup, 0.0)
            g.set_profiling(True)
            g.reset_perf()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.advance(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            pf = g.perf()
            d1 = g.diagnostics()
        out[prec] = {"value": n ** 3 * steps / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / steps,
                     "stage_ms": pf["stage_ms"] / max(1, pf["stage_launches"]),
                     "max_divB_end": d1["max_divB"], "energy_drift_rel": (d1["energy"] - d0["energy"]) / d0["energy"],
                     "mass_drift_rel": (d1["mass"] - d0["mass"]) / d0["mass"]}
    out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def run_euler2d(args, stream, peaks) -> dict:
    """2D Euler/HLLC + gravity (euler2d_gravity_hllc.cpp): (1) the reference's
    own case, init_random_blob (mt19937 seed 42) with its parameters (gamma
    1.2, CFL 0.45, periodic unit square, G 1) and its red-black SOR to the
    residual tolerance 1e-10 (omega 1.7), at --grid-eh; (2) the enclosed-mass
    gravity provider (the rhs's alternative, EH:226-286) on the same IC at
    --grid-eh-enclosed, where the fused stage kernel dominates.  FP64 and FP32."""
    import torch

    from core_collapse_b200.euler2d import Euler2dSolver, ParamsEH, ic_random_blob
    out = {}
    for tag, n, poisson, steps in (("sor", args.grid_eh, "sor", args.steps_eh_sor),
                                   ("enclosed", args.grid_eh_enclosed, "enclosed", args.steps_eh)):
        s0 = ic_random_blob(ParamsEH(Nx=n, Ny=n))
        blk = {"workload": f"Euler/HLLC random blob (seed 42), {n}^2 periodic, "
                           + ("red-black SOR to residual 1e-10" if poisson == "sor" else "enclosed-mass gravity"),
               "steps": steps, "warmup": args.warmup}
        for prec in ("fp32", "fp64"):
            p = ParamsEH(Nx=n, Ny=n, precision=prec, poisson=poisson, t_end=1e30)
            with Euler2dSolver(p) as g:
                g.set_stream(stream.cuda_stream)
                g.upload(s0)
                g.advance(args.warmup, 0.0)
                g.reset_perf()
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                g.advance(steps)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                pf = g.perf()
                d = g.diagnostics()
            blk[prec] = {"value": n * n * steps / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / steps,
                         "gpu_launches": pf["kernel_launches"], "poisson_sweeps_last": d["poisson_iters"],
                         "nonfinite": d["nonfinite"]}
        out[tag] = blk
    return out


# words of FP32/FP64 state moved per cell and Navier-Stokes step: stage 1 reads U,
# phi and writes U1, k1 (13); stage 2 reads U1, U, k1, phi and writes U (17);
# the CFL/density reduction reads U (4) and the stage-2 density sum U1.rho (1);
# each of the two spectral solves reads rho, writes phi and moves the complex
# work array through rows, columns and inverse rows (2 x 10)
NS_STEP_WORDS = 13 + 17 + 4 + 1 + 2 * 10


def run_ns2d(args, stream, peaks) -> dict:
    """2D Navier-Stokes + FFT gravity: the reference's collapse IC (central
    Gaussian overdensity, 1% density noise, Mach-0.05 velocity noise, seed 42)
    and parameters (gamma 1.4, CFL 0.35, mu 1e-6, G 10), periodic unit square."""
    import torch

    from core_collapse_b200.ns2d import Ns2dSolver, ParamsNS, ic_collapse
    n = args.grid_ns
    steps = max(1, min(args.steps, args.steps_ns))
    s0 = ic_collapse(ParamsNS(Nx=n, Ny=n))
    out = {"workload": f"2D Navier-Stokes + spectral gravity, {n}^2 periodic, reference collapse IC and parameters",
           "steps": steps, "warmup": args.warmup, "step_words_per_cell": NS_STEP_WORDS}
    for prec in ("fp32", "fp64"):
        p = ParamsNS(Nx=n, Ny=n, precision=prec, t_end=1e30)
        with Ns2dSolver(p) as g:
            g.set_stream(stream.cuda_stream)
            g.upload(s0)
            d0 = g.diagnostics()
            g.advance(args.warmup, 0.0)
            g.reset_perf()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            g.advance(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            pf = g.perf()
            d1 = g.diagnostics()
        word = 4 if prec == "fp32" else 8
        gbs = NS_STEP_WORDS * word * n * n / (ms / steps / 1000.0) / 1e9
        out[prec] = {"value": n * n * steps / (ms / 1000.0), "unit": UNIT, "ms_per_step": ms / steps,
                     "gpu_launches": pf["kernel_launches"], "step_gbs": gbs,
                     "step_roofline_frac": gbs / peaks["hbm_gbs"],
                     "mass_drift_rel": (d1["mass"] - d0["mass"]) / d0["mass"], "nonfinite": d1["nonfinite"]}
    out["fp32_over_fp64"] = out["fp32"]["value"] / out["fp64"]["value"]
    return out


def run_ensemble(args, stream, rank: int, world: int, barrier, max_over_ranks, single_fp32: float) -> dict:
    """Batched ensemble: 512 independent 2D collapse instances on [-1,1]^2
    with outflow boundaries, side drawn uniformly from {64,96,128,192,256}
    (seed 2), core amplitude U(2,20), width U(0.05,0.2), Bx U(0,0.2), eta
    log-uniform [1e-4,1e-2]; gamma 5/3, G 1, CFL 0.4, direct Poisson; FP32
    state, FP32 Poisson solve and FP64 reductions.  Instances are split over
    the ranks by cell count (no collective inside a step).  The single-grid
    comparison runs one large instance of the same physics and Poisson kind
    (--ensemble-single-side^2, outflow, direct solve) through the same handle
    type for the same number of steps."""
    import numpy as np
    import torch

    from core_collapse_b200.batch import BatchSolver, collapse_ensemble, partition_by_cells
    from core_collapse_b200.mhd2d import ic_collapse
    params, states = collapse_ensemble(args.ensemble, seed=2, precision="fp32")
    mine = partition_by_cells(params, world)[rank]
    total_cells = sum(p.Nx * p.Ny for p in params)
    steps = max(1, args.ensemble_steps)
    out = {"workload": f"{args.ensemble} independent 2D collapse instances, sides from {{64,96,128,192,256}} (seed 2), "
                       "outflow [-1,1]^2, per-instance core amplitude/width, Bx, eta; direct Poisson",
           "instances": args.ensemble, "cells": total_cells, "steps": steps, "warmup": args.warmup,
           "dtype": "f32", "reductions": "f64", "poisson": "direct (FP32, the instances' precision)", "scaling": "strong"}
    b = BatchSolver([params[i] for i in mine])
    b.set_stream(stream.cuda_stream)
    for k, i in enumerate(mine):
        b.upload(k, *states[i])
    shape, tune_ms = b.autotune(reps=3)
    b.advance(args.warmup, np.zeros(len(mine)))
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.advance(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    info = b.info()
    nonfinite = sum(b.diagnostics(k)["nonfinite"] for k in range(len(mine)))
    # share of the stage kernels in a step, from profiled stage events (eager, no graph)
    b.set_profiling(True)
    b.reset_perf()
    e0.record(stream)
    b.advance(3)
    e1.record(stream)
    torch.cuda.synchronize()
    pf = b.perf()
    b.close()
    value = total_cells * steps / (ms / 1000.0)

    # one large instance, same physics and Poisson kind (rank-local, no collective)
    from dataclasses import replace as dc_replace
    ns = args.ensemble_single_side
    p1 = dc_replace(params[0], Nx=ns, Ny=ns, eta=1e-3)
    U1, B1 = ic_collapse(p1, core_amp=9.0, core_width=0.1, noise=0.01, seed=0, Bx0=0.05)
    with BatchSolver([p1]) as b1:
        b1.set_stream(stream.cuda_stream)
        b1.upload(0, U1, B1)
        b1.autotune(reps=3)
        b1.advance(args.warmup, np.zeros(1))
        torch.cuda.synchronize()
        e0.record(stream)
        b1.advance(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        single_value = ns * ns * steps / (e0.elapsed_time(e1) / 1000.0)

    # batching efficiency of the step machinery alone: the same ensemble and one
    # large instance, both without gravity (the direct solve's cost per cell
    # grows with the side, so with gravity a large grid is slower per cell)
    def timed_batch(plist, slist, nsteps):
        with BatchSolver(plist) as bb:
            bb.set_stream(stream.cuda_stream)
            for kk, st_ in enumerate(slist):
                bb.upload(kk, *st_)
            bb.autotune(reps=3)
            bb.advance(args.warmup, np.zeros(len(plist)))
            torch.cuda.synchronize()
            e0.record(stream)
            bb.advance(nsteps)
            e1.record(stream)
            torch.cuda.synchronize()
            return sum(q.Nx * q.Ny for q in plist) * nsteps / (e0.elapsed_time(e1) / 1000.0)

    ng_steps = max(1, min(steps, 60))
    ens_nograv = timed_batch([dc_replace(params[i], gravity_on=False) for i in mine], [states[i] for i in mine],
                             ng_steps)
    big = args.ensemble_nograv_side
    pb = dc_replace(params[0], Nx=big, Ny=big, eta=1e-3, gravity_on=False)
    single_nograv = timed_batch([pb], [ic_collapse(pb, core_amp=9.0, core_width=0.1, noise=0.01, seed=0, Bx0=0.05)],
                                ng_steps)
    out.update({"value": value, "unit": UNIT, "ms_per_step": ms / steps,
                "single_grid": {"workload": f"one {ns}^2 collapse instance (core 9, width 0.1, Bx 0.05, eta 1e-3), "
                                            "outflow, direct Poisson, FP32, same handle type",
                                "value": single_value, "unit": UNIT},
                "ensemble_over_single_grid": value / world / single_value,
                "ensemble_over_single_fft_grid": value / world / single_fp32 if single_fp32 else None,
                "no_gravity": {"steps": ng_steps, "ensemble_value": ens_nograv,
                               "single_grid": f"one {big}^2 instance, same handle type",
                               "single_value": single_nograv, "ensemble_over_single_grid": ens_nograv / single_nograv},
                "tile": [info["tile_x"], info["tile_y"]], "autotune_choice": shape, "autotune_stage_ms": tune_ms,
                "stage_ctas": info["stage_ctas"], "stage_tiles": info["stage_tiles"],
                # stage-kernel time per step (events around the stage launches of 3 eager
                # steps) over the graph-timed step
                "stage_share_of_step": (pf["stage_ms"] / 3.0) / (ms / steps) if ms > 0 else None,
                "nonfinite_instances": nonfinite, "device_bytes_rank0": info["device_bytes"]})
    return out


# per-entry finite-difference errors are reported for entries whose central
# difference exceeds this fraction of the largest gradient: below it the
# difference quotient's own roundoff (~1e-16 |loss| / h) dominates
ADJ_FD_FLOOR = 1e-2


def run_adjoint(args, stream) -> dict:
    """Discrete adjoint of the 2D step: 512^2 collapse on [-1,1]^2 with
    outflow boundaries (gamma 5/3, G 1, eta 1e-3, CFL 0.4, direct Poisson),
    core amplitude 9, width 0.1, 1% density noise (seed 0), Bx 0.05; 100
    steps, a checkpoint every 10.  Loss 0.5 sum (rho_T - rho_target)^2, the
    target from the same run with core amplitude 12 (seed 3).  FP64, and an
    FP32 forward with FP32 reverse kernels beside it.
    Reported: recorded-forward and VJP times (CUDA events on the handle's
    stream), their ratio, and central finite differences (h 1e-6, recorded
    dt replayed) of the loss along --adjoint-fd random cell directions (FP64);
    for FP32 the gradient's distance from the FP64 one."""
    import numpy as np
    import torch

    from core_collapse_b200.adjoint import AdjointSolver, density_loss_adjoint
    from core_collapse_b200.mhd2d import Params, ic_collapse
    n, nsteps, k = args.adjoint_grid, args.adjoint_steps, 10
    p = Params(Nx=n, Ny=n, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=False, periodic_y=False, gamma=5.0 / 3.0,
               G=1.0, eta=1e-3, cfl=0.4, gravity_on=True, poisson="direct", precision="fp64", t_end=1e30)
    U, B = ic_collapse(p, core_amp=9.0, core_width=0.1, noise=0.01, seed=0, Bx0=0.05)
    Ut, Bt = ic_collapse(p, core_amp=12.0, core_width=0.1, noise=0.01, seed=3, Bx0=0.05)
    out = {"workload": f"{n}^2 collapse, outflow [-1,1]^2, gamma 5/3, G 1, eta 1e-3, CFL 0.4, direct Poisson, "
                       f"{nsteps} steps, checkpoint every {k}; loss 0.5 |rho_T - rho_target|^2 (target: core 12, seed 3)",
           "dtype": "f64"}
    with AdjointSolver(p, k, nsteps) as s:
        s.set_stream(stream.cuda_stream)
        s.upload(Ut, Bt)
        s.forward(nsteps)
        target = s.download()[0].rho.copy()
        s.upload(U, B)
        s.forward(nsteps)                       # warm-up (and the recorded dt)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record(stream)
        s.forward(nsteps)
        e1.record(stream)
        UT, _ = s.download()
        loss, lamU, lamB = density_loss_adjoint(p, UT.rho, target)
        torch.cuda.synchronize()
        e1.synchronize()
        e2.record(stream)
        g, _, geta = s.vjp(lamU, lamB)
        e3 = torch.cuda.Event(enable_timing=True)
        e3.record(stream)
        torch.cuda.synchronize()
        fwd_ms, adj_ms = e0.elapsed_time(e1), e2.elapsed_time(e3)
        rng = np.random.default_rng(3)
        cells = rng.choice(n * n, size=args.adjoint_fd, replace=False)
        worst = 0.0
        gscale = float(np.max(np.abs(g.rho)))
        floor = ADJ_FD_FLOOR * gscale
        per_entry, n_above = 0.0, 0
        for c in cells:
            vals = []
            for sgn in (1.0, -1.0):
                V = U.copy()
                V.rho[c] += sgn * 1e-6
                s.upload(V, B)
                s.forward(nsteps, replay=True)
                vals.append(density_loss_adjoint(p, s.download()[0].rho, target)[0])
            fd = (vals[0] - vals[1]) / 2e-6
            worst = max(worst, abs(g.rho[c] - fd) / gscale)
            if abs(fd) > floor:
                n_above += 1
                per_entry = max(per_entry, abs(g.rho[c] - fd) / abs(fd))
    out.update({"forward_ms": fwd_ms, "adjoint_ms": adj_ms, "adjoint_over_forward": adj_ms / fwd_ms,
                "zone_updates_per_s_forward": n * n * nsteps / (fwd_ms / 1000.0),
                "loss": loss, "dloss_deta": geta,
                "fd_check": {"cells": int(args.adjoint_fd), "h": 1e-6,
                             "max_abs_err_over_max_grad": worst,
                             "max_rel_err_per_entry": per_entry, "entries_above_floor": n_above,
                             "floor": f"|fd| > {ADJ_FD_FLOOR:g} x max|grad|"}})
    # the same workload with an FP32 forward and FP32 reverse kernels; its
    # gradient against the FP64 one (a finite difference of an FP32 map
    # measures rounding), the same target density
    from dataclasses import replace as dc_replace
    g64 = g.rho.copy()
    with AdjointSolver(dc_replace(p, precision="fp32"), k, nsteps) as s:
        s.set_stream(stream.cuda_stream)
        s.upload(U, B)
        s.forward(nsteps)                       # warm-up (and the recorded dt)
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        torch.cuda.synchronize()
        e0.record(stream)
        s.forward(nsteps)
        e1.record(stream)
        UT, _ = s.download()
        loss32, lamU, lamB = density_loss_adjoint(p, UT.rho, target)
        torch.cuda.synchronize()
        e2.record(stream)
        g32, _, geta32 = s.vjp(lamU, lamB)
        e3.record(stream)
        torch.cuda.synchronize()
        f32, a32 = e0.elapsed_time(e1), e2.elapsed_time(e3)
    # the same workload with the single-grid red-black SOR instead of the direct
    # solve (the reference M2's fixed 600 sweeps, omega 1.9), FP64
    with AdjointSolver(dc_replace(p, poisson="sor", sor_iters=args.adjoint_sor_sweeps, sor_omega=1.9), k,
                       nsteps) as s:
        s.set_stream(stream.cuda_stream)
        s.upload(U, B)
        s.forward(nsteps)
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        torch.cuda.synchronize()
        e0.record(stream)
        s.forward(nsteps)
        e1.record(stream)
        UT, _ = s.download()
        loss_s, lamU, lamB = density_loss_adjoint(p, UT.rho, target)
        torch.cuda.synchronize()
        e2.record(stream)
        gs, _, geta_s = s.vjp(lamU, lamB)
        e3.record(stream)
        torch.cuda.synchronize()
        fs, as_ = e0.elapsed_time(e1), e2.elapsed_time(e3)
    out["sor"] = {"forward_ms": fs, "adjoint_ms": as_, "adjoint_over_forward": as_ / fs, "loss": loss_s,
                  "dloss_deta": geta_s, "sweeps_per_solve": args.adjoint_sor_sweeps,
                  "note": "red-black SOR gravity (omega 1.9, fixed sweeps), reversed sweep by sweep; FP64"}
    out["fp32"] = {"forward_ms": f32, "adjoint_ms": a32, "adjoint_over_forward": a32 / f32,
                   "zone_updates_per_s_forward": n * n * nsteps / (f32 / 1000.0), "loss": loss32,
                   "dloss_deta": geta32,
                   "grad_vs_fp64_max_abs_err_over_max_grad": float(np.max(np.abs(g32.rho - g64)) / gscale),
                   "note": "FP32 forward, FP32 reverse kernels (eta adjoint summed in FP64); own CFL dt"}
    return out


def run_ensemble_only(args) -> None:
    import torch
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    print(json.dumps(run_ensemble(args, stream, 0, 1, torch.cuda.synchronize, lambda x: x, 0.0)), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--grid", type=int, default=4096)
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--cpu-sample-grid", type=int, default=512)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--stage-kernel", choices=["march", "tile"], default="tile",
                    help="FP32 stage kernel of the headline run")
    ap.add_argument("--march-rows", type=int, default=0, help="rows per march segment (0: from the grid)")
    ap.add_argument("--skip-ladder", action="store_true")
    ap.add_argument("--ladder-steps", type=int, default=500)
    ap.add_argument("--ladder-grids", default="1024,4096")
    ap.add_argument("--skip-3d", action="store_true")
    ap.add_argument("--grid3d", type=int, default=256)
    ap.add_argument("--steps3d", type=int, default=100)
    ap.add_argument("--skip-ns", action="store_true")
    ap.add_argument("--skip-eh", action="store_true")
    ap.add_argument("--grid-eh", type=int, default=512)
    ap.add_argument("--steps-eh-sor", type=int, default=1)
    ap.add_argument("--grid-eh-enclosed", type=int, default=4096)
    ap.add_argument("--steps-eh", type=int, default=20)
    ap.add_argument("--eh-only", action="store_true", help="time only the Euler/HLLC block (a profiling aid)")
    ap.add_argument("--grid-ns", type=int, default=4096)
    ap.add_argument("--steps-ns", type=int, default=20)
    ap.add_argument("--skip-ensemble", action="store_true")
    ap.add_argument("--ensemble", type=int, default=512)
    ap.add_argument("--ensemble-steps", type=int, default=300)
    ap.add_argument("--ensemble-single-side", type=int, default=2048)
    ap.add_argument("--ensemble-nograv-side", type=int, default=4096)
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--adjoint-grid", type=int, default=512)
    ap.add_argument("--adjoint-steps", type=int, default=100)
    ap.add_argument("--adjoint-fd", type=int, default=64)
    ap.add_argument("--adjoint-sor-sweeps", type=int, default=600)
    ap.add_argument("--adjoint-only", action="store_true", help="time only the adjoint block (a profiling aid)")
    ap.add_argument("--ns-only", action="store_true",
                    help="time only the Navier-Stokes block (a profiling aid; prints the ns2d block)")
    ap.add_argument("--ensemble-only", action="store_true",
                    help="time only the batched ensemble (a profiling aid; prints the ensemble block)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.ensemble_only:
        run_ensemble_only(args)
        return
    if args.eh_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_euler2d(args, torch.cuda.Stream(), measured_peaks())), flush=True)
        return
    if args.ns_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_ns2d(args, torch.cuda.Stream(), measured_peaks())), flush=True)
        return
    if args.adjoint_only:
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_adjoint(args, torch.cuda.Stream())), flush=True)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
