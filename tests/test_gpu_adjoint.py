"""GPU checks of the discrete adjoint of the 2D MHD step (cc_adjoint_*).

The adjoint is the exact transpose of the recorded discrete map (dt of each
step recorded, then held fixed), so it is checked against central finite
differences of the same map (replayed dt): directional derivatives of all
eight state fields along random directions, single-cell density gradients of
the density misfit loss, and the eta gradient through a second handle that
replays the recorded dt.  Tolerance: 1e-6 relative.  Test states keep every
face off the HLL branch (Bn != 0) and every MC slope off its zero kink, so a
finite-difference step measures a derivative, not a branch jump."""
import ctypes as C

import numpy as np
import pytest

import oracle_lib as O

from core_collapse_b200.adjoint import AdjointSolver, Mhd2dRollout, RolloutSetup, density_loss_adjoint
from cases_adjoint import make_case_adj as _case
from core_collapse_b200.mhd2d import empty_state

pytestmark = pytest.mark.gpu

FIELDS = ["rho", "mx", "my", "mz", "E", "Bz", "Bx_f", "By_f"]


def _arrays(U, B):
    return U.arrays() + [B.Bx_f, B.By_f]


def _combine(U, B, dU, dB, h):
    V, W = U.copy(), B.copy()
    for a, d in zip(_arrays(V, W), _arrays(dU, dB)):
        a += h * d
    return V, W


def _run(s, U, B, nsteps, replay):
    s.upload(U, B)
    s.forward(nsteps, 0.0, replay=replay)
    return s.download()


@pytest.mark.parametrize("periodic,grav", [(False, True), (True, True), (True, False)])
def test_directional_derivative_all_fields(periodic, grav):
    p, U, B = _case(periodic, grav)
    nsteps = 7
    rng = np.random.default_rng(5)
    with AdjointSolver(p, checkpoint_every=3, max_steps=nsteps) as s:
        _run(s, U, B, nsteps, replay=False)
        lamU, lamB = empty_state(p)
        for a in _arrays(lamU, lamB):
            a[:] = rng.normal(size=a.size)
        l0U, l0B, _ = s.vjp(lamU, lamB)
        dU, dB = empty_state(p)
        for a, ref in zip(_arrays(dU, dB), _arrays(U, B)):
            a[:] = rng.normal(size=a.size) * (np.abs(ref).mean() + 1e-3)
        adj = sum(float(x @ v) for x, v in zip(_arrays(l0U, l0B), _arrays(dU, dB)))
        # a step moving all ~5000 inputs at once: at 1e-6 a limiter or floor
        # branch point of some cell falls inside the step in longer runs; at
        # 1e-7 none does, and roundoff stays below 1e-8 of the derivative
        h = 1e-7
        Up, Bp = _run(s, *_combine(U, B, dU, dB, h), nsteps, replay=True)
        Um, Bm = _run(s, *_combine(U, B, dU, dB, -h), nsteps, replay=True)
        fd = sum(float(l @ (a - b)) for l, a, b in zip(_arrays(lamU, lamB), _arrays(Up, Bp), _arrays(Um, Bm))) / (2 * h)
    assert abs(adj - fd) <= 1e-6 * abs(fd), f"adjoint {adj} vs finite differences {fd}"


def test_density_gradient_cells_and_eta():
    p, U, B = _case(False, True)
    nsteps = 6
    _, T, _ = _case(False, True, seed=9)   # a target density
    with AdjointSolver(p, checkpoint_every=4, max_steps=nsteps) as s:
        UT, BT = _run(s, U, B, nsteps, replay=False)
        dts = s.dts()
        loss0, lamU, lamB = density_loss_adjoint(p, UT.rho, T.rho)
        g0, _, geta = s.vjp(lamU, lamB)
        rng = np.random.default_rng(1)
        cells = rng.choice(p.Nx * p.Ny, size=8, replace=False)
        h = 1e-6
        for c in cells:
            Vp, Vm = U.copy(), U.copy()
            Vp.rho[c] += h
            Vm.rho[c] -= h
            lp = density_loss_adjoint(p, _run(s, Vp, B, nsteps, True)[0].rho, T.rho)[0]
            lm = density_loss_adjoint(p, _run(s, Vm, B, nsteps, True)[0].rho, T.rho)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(g0.rho[c] - fd) <= 1e-6 * np.max(np.abs(g0.rho)), f"cell {c}: {g0.rho[c]} vs {fd}"
    # eta: two more handles replaying the same dt sequence; the absolute step
    # 1e-6 balances roundoff of the loss against truncation
    de = 1e-6
    losses = []
    for e in (p.eta + de, p.eta - de):
        from dataclasses import replace
        with AdjointSolver(replace(p, eta=e), checkpoint_every=4, max_steps=nsteps) as s2:
            s2.set_dts(dts)
            losses.append(density_loss_adjoint(p, _run(s2, U, B, nsteps, True)[0].rho, T.rho)[0])
    fd_eta = (losses[0] - losses[1]) / (2 * de)
    assert abs(geta - fd_eta) <= 1e-6 * abs(fd_eta), f"eta: {geta} vs {fd_eta}"


def test_checkpoint_interval_does_not_change_the_gradient():
    p, U, B = _case(True, True)
    nsteps = 7
    out = []
    for k in (1, 3, 7):
        with AdjointSolver(p, checkpoint_every=k, max_steps=nsteps) as s:
            UT, _ = _run(s, U, B, nsteps, replay=False)
            _, lamU, lamB = density_loss_adjoint(p, UT.rho, np.ones_like(UT.rho))
            g, gB, ge = s.vjp(lamU, lamB)
            out.append((g.rho.copy(), gB.Bx_f.copy(), ge))
    for g, gb, ge in out[1:]:
        assert np.max(np.abs(g - out[0][0])) <= 1e-12 * np.max(np.abs(out[0][0]))
        assert np.max(np.abs(gb - out[0][1])) <= 1e-12 * np.max(np.abs(out[0][1])) + 1e-300
        assert abs(ge - out[0][2]) <= 1e-12 * abs(out[0][2])


def test_autograd_function_matches_the_c_abi():
    torch = pytest.importorskip("torch")
    p, U, B = _case(False, True)
    setup = RolloutSetup(params=p, U0=U, B0=B, nsteps=4, checkpoint_every=2)
    rho0 = torch.tensor(U.rho, dtype=torch.float64, requires_grad=True)
    eta = torch.tensor(p.eta, dtype=torch.float64, requires_grad=True)
    rhoT = Mhd2dRollout.apply(rho0, eta, setup)
    target = torch.ones_like(rhoT)
    loss = 0.5 * ((rhoT - target) ** 2).sum()
    loss.backward()
    with AdjointSolver(p, checkpoint_every=2, max_steps=4) as s:
        UT, _ = _run(s, U, B, 4, replay=False)
        _, lamU, lamB = density_loss_adjoint(p, UT.rho, np.ones_like(UT.rho))
        g, _, ge = s.vjp(lamU, lamB)
    assert np.allclose(rho0.grad.numpy(), g.rho, rtol=1e-12, atol=1e-14 * np.abs(g.rho).max())
    assert abs(eta.grad.item() - ge) <= 1e-12 * abs(ge)


@pytest.mark.parametrize("periodic,grav", [(False, True), (True, True), (True, False)])
def test_adjoint_is_the_transpose_of_the_dual_number_tangent(periodic, grav):
    """<lambda_T, J v> from the oracle's dual-number tangent-linear build
    (same recorded dt) equals <J^T lambda_T, v> from the GPU adjoint, and the
    GPU forward equals the oracle's value trajectory bit for bit."""
    p, U, B = _case(periodic, grav)
    nsteps = 5
    rng = np.random.default_rng(21)
    with AdjointSolver(p, checkpoint_every=2, max_steps=nsteps) as s:
        UT, BT = _run(s, U, B, nsteps, replay=False)
        dts = s.dts()
        lamU, lamB = empty_state(p)
        for a in _arrays(lamU, lamB):
            a[:] = rng.normal(size=a.size)
        l0U, l0B, _ = s.vjp(lamU, lamB)
    V = [rng.normal(size=a.size) * (np.abs(a).mean() + 1e-3) for a in _arrays(U, B)]
    vals = O.copy_state(_arrays(U, B))
    tans = O.copy_state(V)
    cp = p.to_c()
    assert O.oracle().or_mhd2d_tlm(C.byref(cp), O.pp(vals), O.pp(tans), nsteps, O.dp(dts)) == 0
    for a, b in zip(vals, _arrays(UT, BT)):
        assert np.array_equal(a, b)
    lhs = sum(float(l @ t) for l, t in zip(_arrays(lamU, lamB), tans))
    rhs = sum(float(l @ v) for l, v in zip(_arrays(l0U, l0B), V))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs), f"<lam, Jv> {lhs} vs <J^T lam, v> {rhs}"
