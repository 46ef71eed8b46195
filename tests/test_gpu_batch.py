"""GPU parity of the batched 2D MHD ensemble (cc_batch_*).

FP64: every instance of a mixed batch (sizes, boundary kinds, gravity on and
off, its own eta, CFL and t_end) reproduces the oracle's main loop with the
direct Poisson solve (oracle mode 3) bit for bit; without gravity it also
equals the single-grid solver bit for bit.  The direct solve itself equals
the SOR's converged solution to roundoff (CPU pin in test_oracle_direct.py).
Any instance's result is independent of the rest of the batch and of the
stage tile shape (bitwise, FP64 and FP32)."""
import ctypes as C
from dataclasses import replace

import numpy as np
import pytest

import oracle_lib as O
from core_collapse_b200 import _lib as L
from core_collapse_b200.batch import BatchSolver, collapse_ensemble
from core_collapse_b200.mhd2d import CcError, Mhd2dSolver, Params, ic_collapse, ic_orszag_tang

pytestmark = pytest.mark.gpu


def _mixed(precision="fp64"):
    """Five instances covering both boundary kinds per axis, gravity on/off,
    eta 0 and > 0, uneven sizes and tile remainders."""
    base = Params(x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, gamma=5.0 / 3.0, cfl=0.4, G=1.0, poisson="direct",
                  precision=precision, t_end=10.0)
    specs = [
        (dict(Nx=40, Ny=24, periodic_x=False, periodic_y=False, eta=1e-3, gravity_on=True), "collapse", 9.0, 0.3, 1),
        (dict(Nx=16, Ny=36, periodic_x=True, periodic_y=True, eta=5e-4, gravity_on=True), "collapse", 4.0, 0.25, 2),
        (dict(Nx=33, Ny=20, periodic_x=False, periodic_y=True, eta=2e-3, gravity_on=True), "collapse", 6.0, 0.4, 3),
        (dict(Nx=24, Ny=18, periodic_x=True, periodic_y=False, eta=0.0, gravity_on=False), "ot", 4.0, 0.3, 4),
        (dict(Nx=12, Ny=12, periodic_x=True, periodic_y=False, eta=1e-3, gravity_on=True, G=3.0), "collapse", 12.0, 0.35, 5),
    ]
    params, states = [], []
    for kw, kind, amp, width, seed in specs:
        p = replace(base, **kw)
        if kind == "collapse":
            U, B = ic_collapse(p, core_amp=amp, core_width=width, noise=0.02, seed=seed, Bx0=0.05 * seed)
        else:
            U, B = ic_orszag_tang(p, core_amp=amp, core_width=width)
        params.append(p)
        states.append((U, B))
    return params, states


def _run_batch(params, states, nsteps, shape=None, t=None):
    with BatchSolver(params) as b:
        if shape is not None:
            b.set_shape(shape)
        for i, (U, B) in enumerate(states):
            b.upload(i, U, B)
        tt = b.advance(nsteps, np.zeros(len(params)) if t is None else t)
        out = [b.download(i) for i in range(len(params))]
        diags = [b.diagnostics(i) for i in range(len(params))]
    return out, tt, diags


def _flat(U, B):
    return U.arrays() + [B.Bx_f, B.By_f]


def test_fp64_batch_equals_oracle_direct_bitwise():
    params, states = _mixed("fp64")
    out, tt, diags = _run_batch(params, states, 4)   # 3 graph-captured steps + 1 eager
    for i, p in enumerate(params):
        want, tw = O.m2_main_loop_oracle(p.to_c(), O.state_list(*states[i]), 4, mode=3)
        assert tt[i] == tw, f"instance {i}: t {tt[i]} != {tw}"
        assert diags[i]["steps"] == 4
        for k, (a, w) in enumerate(zip(_flat(*out[i]), want)):
            assert np.array_equal(a, w), f"instance {i} field {k}: max |d| {np.max(np.abs(a - w))}"


def test_compute_dt_matches_oracle():
    params, states = _mixed("fp64")
    with BatchSolver(params) as b:
        for i, (U, B) in enumerate(states):
            b.upload(i, U, B)
        dt = b.compute_dt()
    for i, p in enumerate(params):
        assert dt[i] == O.oracle().or_mhd2d_compute_dt(C.byref(p.to_c()), O.pp(O.state_list(*states[i])))


def test_no_gravity_instance_equals_single_grid_bitwise():
    params, states = _mixed("fp64")
    out, tt, _ = _run_batch(params, states, 5)
    i = 3
    p = params[i]
    with Mhd2dSolver(replace(p, poisson="sor")) as s:
        s.upload(*states[i])
        t = s.advance(5, 0.0)
        U, B = s.download()
    assert t == tt[i]
    for a, w in zip(_flat(*out[i]), _flat(U, B)):
        assert np.array_equal(a, w)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_instance_independent_of_batch_and_tile_shape(precision):
    params, states = _mixed(precision)
    with BatchSolver(params) as b:
        nshape = b.info()["n_shapes"]
    ref, tref, _ = _run_batch(params, states, 4, shape=0)
    for shape in range(1, nshape):
        out, tt, _ = _run_batch(params, states, 4, shape=shape)
        assert np.array_equal(tt, tref)
        for i in range(len(params)):
            for a, w in zip(_flat(*out[i]), _flat(*ref[i])):
                assert np.array_equal(a, w), f"shape {shape} instance {i}"
    for i in (0, 2):
        alone, ta, _ = _run_batch([params[i]], [states[i]], 4)
        assert ta[0] == tref[i]
        for a, w in zip(_flat(*alone[0]), _flat(*ref[i])):
            assert np.array_equal(a, w), f"instance {i} alone differs"


def test_instances_stop_at_their_own_t_end():
    params, states = _mixed("fp64")
    params[1] = replace(params[1], t_end=0.004)
    params[4] = replace(params[4], t_end=0.0)
    out, tt, diags = _run_batch(params, states, 6)
    assert tt[1] == 0.004 and tt[4] == 0.0 and diags[4]["steps"] == 0
    for i, p in enumerate(params):
        want, tw = O.m2_main_loop_oracle(p.to_c(), O.state_list(*states[i]), 6, mode=3)
        assert tt[i] == tw
        for a, w in zip(_flat(*out[i]), want):
            assert np.array_equal(a, w), f"instance {i}"


def test_fp32_batch_error_vs_fp64_oracle():
    """FP32 bulk arithmetic with FP64 reductions and FP64 Poisson: per-field
    relative L1 error against the FP64 oracle after 20 steps below 1e-5."""
    params, states = _mixed("fp32")
    out, tt, _ = _run_batch(params, states, 20)
    for i, p in enumerate(params):
        want, tw = O.m2_main_loop_oracle(replace(p, precision="fp64").to_c(), O.state_list(*states[i]), 20, mode=3)
        assert abs(tt[i] - tw) <= 1e-5 * tw
        for k, (a, w) in enumerate(zip(_flat(*out[i]), want)):
            scale = np.mean(np.abs(w)) + 1e-30
            l1 = np.mean(np.abs(a - w)) / scale
            assert l1 <= 1e-5, f"instance {i} field {k}: rel L1 {l1:.2e}"


def test_fp32_tensor_core_poisson_vs_fp64_oracle():
    """FP32 instances whose Nx are multiples of 4 solve the direct Poisson
    transforms on the tcgen05 tensor cores (3xTF32, 128 x 128 tiles): sizes
    with one and several tiles and partial tiles, both boundary kinds; per-field
    relative L1 error against the FP64 oracle after 10 steps below 1e-5 (the
    face fields relative to the mean in-plane field |Bx_f| + |By_f|: By_f
    starts at zero and stays small, so its own mean is no scale)."""
    base = Params(x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, gamma=5.0 / 3.0, cfl=0.4, G=1.0, poisson="direct",
                  precision="fp32", t_end=10.0, gravity_on=True)
    specs = [dict(Nx=40, Ny=24, periodic_x=False, periodic_y=False, eta=1e-3),
             dict(Nx=136, Ny=200, periodic_x=True, periodic_y=True, eta=5e-4),
             dict(Nx=260, Ny=132, periodic_x=False, periodic_y=True, eta=2e-3),
             dict(Nx=128, Ny=128, periodic_x=True, periodic_y=False, eta=1e-3)]
    params, states = [], []
    for k, kw in enumerate(specs):
        p = replace(base, **kw)
        U, B = ic_collapse(p, core_amp=6.0 + 2 * k, core_width=0.25, noise=0.02, seed=11 + k, Bx0=0.05)
        params.append(p)
        states.append((U, B))
    with BatchSolver(params) as b:
        assert b.info()["poisson_tile"] == 128
    out, tt, _ = _run_batch(params, states, 10)
    for i, p in enumerate(params):
        want, tw = O.m2_main_loop_oracle(replace(p, precision="fp64").to_c(), O.state_list(*states[i]), 10, mode=3)
        assert abs(tt[i] - tw) <= 1e-5 * tw
        bscale = np.mean(np.abs(want[6])) + np.mean(np.abs(want[7]))
        for k, (a, w) in enumerate(zip(_flat(*out[i]), want)):
            scale = (bscale if k >= 6 else np.mean(np.abs(w))) + 1e-30
            l1 = np.mean(np.abs(a - w)) / scale
            assert l1 <= 1e-5, f"instance {i} field {k}: rel L1 {l1:.2e}"


def test_mass_conserved_periodic_instance():
    params, states = _mixed("fp64")
    out, tt, diags = _run_batch(params, states, 6)
    U0, _ = states[1]
    dV = params[1].dx * params[1].dy
    m0 = U0.rho.sum() * dV
    assert abs(diags[1]["mass"] - m0) <= 1e-13 * m0
    assert diags[1]["max_divB"] < 1e-10


def test_autotune_and_collapse_ensemble():
    params, states = collapse_ensemble(12, seed=2, sides=(32, 48, 64), precision="fp32")
    with BatchSolver(params) as b:
        for i, (U, B) in enumerate(states):
            b.upload(i, U, B)
        shape, ms = b.autotune(reps=2)
        info = b.info()
        assert info["shape"] == shape and ms > 0
        assert info["cells"] == sum(p.Nx * p.Ny for p in params)
        t = b.advance(3, np.zeros(len(params)))
        assert np.all(t > 0)
        for i in range(len(params)):
            d = b.diagnostics(i)
            assert d["nonfinite"] == 0 and d["steps"] == 3


def test_create_rejects_sor_gravity():
    p = Params(Nx=16, Ny=16, gravity_on=True, poisson="sor")
    with pytest.raises(CcError) as e:
        BatchSolver([p])
    assert e.value.code == L.CC_ERR_UNSUPPORTED


def test_times_equal_diagnostics():
    """cc_batch_times (one copy of the device clocks) == each instance's
    diagnostics time after advance(nsteps) without start times."""
    from core_collapse_b200.batch import BatchSolver, collapse_ensemble
    params, states = collapse_ensemble(6, seed=5, precision="fp64")
    with BatchSolver(params) as b:
        for k in range(len(params)):
            b.upload(k, *states[k])
        t = b.advance(3)
        want = np.array([b.diagnostics(i)["t"] for i in range(len(params))])
        assert np.array_equal(t, want) and np.array_equal(b.times(), want) and np.all(want > 0)
