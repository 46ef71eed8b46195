"""The discrete adjoint with SOR gravity (cc_adjoint_create with poisson_kind
CC_POISSON_SOR): the forward solve is the single-grid solver's red-black SOR
(M2:178-237 in red-black order, sor_iters sweeps), reversed sweep by sweep
with each solve's sweep count.

Checked: the adjoint handle's forward run equals the single-grid handle's main
loop (same SOR) to 1e-12; central finite differences (h 1e-6, recorded dt
replayed) of the density-misfit loss at single cells and of the
final-state inner product along a random direction of all eight fields
agree with the VJP to 1e-6 relative; and the eta derivative (step 1e-7)."""
import numpy as np
import pytest

import oracle_lib as O
from cases_adjoint import make_case_adj
from core_collapse_b200.adjoint import AdjointSolver, density_loss_adjoint
from core_collapse_b200.mhd2d import Mhd2dSolver

pytestmark = pytest.mark.gpu


def _case(periodic, seed=3):
    from dataclasses import replace
    p, U, B = make_case_adj(periodic, True, seed=seed)
    return replace(p, poisson="sor", sor_iters=60, sor_omega=1.8), U, B


def _run(s, U, B, nsteps, replay):
    s.upload(U, B)
    s.forward(nsteps, 0.0, replay=replay)
    return s.download()


@pytest.mark.parametrize("periodic", [False, True])
def test_sor_adjoint_forward_matches_single_grid(periodic):
    from dataclasses import replace
    p, U, B = _case(periodic)
    n = 4
    with AdjointSolver(p, checkpoint_every=2, max_steps=n) as s:
        got = O.state_list(*_run(s, U, B, n, False))
    with Mhd2dSolver(replace(p, t_end=1e30)) as g:
        g.upload(U, B)
        g.advance(n, 0.0)
        want = O.state_list(*g.download())
    worst = max(O.rel_linf(a, b) for a, b in zip(got, want))
    assert worst <= 1e-12, worst


@pytest.mark.parametrize("periodic", [False, True])
def test_sor_adjoint_density_gradient_and_direction(periodic):
    from dataclasses import replace
    p, U, B = _case(periodic)
    _, T, _ = _case(periodic, seed=9)
    nsteps = 5
    with AdjointSolver(p, checkpoint_every=2, max_steps=nsteps) as s:
        UT, BT = _run(s, U, B, nsteps, False)
        dts = s.dts()
        loss0, lamU, lamB = density_loss_adjoint(p, UT.rho, T.rho)
        g0, gB0, geta = s.vjp(lamU, lamB)
        rng = np.random.default_rng(1)
        h = 1e-6
        for c in rng.choice(p.Nx * p.Ny, size=6, replace=False):
            Vp, Vm = U.copy(), U.copy()
            Vp.rho[c] += h
            Vm.rho[c] -= h
            lp = density_loss_adjoint(p, _run(s, Vp, B, nsteps, True)[0].rho, T.rho)[0]
            lm = density_loss_adjoint(p, _run(s, Vm, B, nsteps, True)[0].rho, T.rho)[0]
            fd = (lp - lm) / (2 * h)
            assert abs(g0.rho[c] - fd) <= 1e-6 * np.max(np.abs(g0.rho)), f"cell {c}: {g0.rho[c]} vs {fd}"
        # all fields along one random direction (faces included)
        dU, dB = U.copy(), B.copy()
        for a in dU.arrays() + [dB.Bx_f, dB.By_f]:
            a[:] = rng.normal(0.0, 1.0, a.size) * (1e-3 * np.max(np.abs(a)) + 1e-6)
        Vp, Wp, Vm, Wm = U.copy(), B.copy(), U.copy(), B.copy()
        for a, b, d in zip(Vp.arrays() + [Wp.Bx_f, Wp.By_f], Vm.arrays() + [Wm.Bx_f, Wm.By_f],
                           dU.arrays() + [dB.Bx_f, dB.By_f]):
            a += h * d
            b -= h * d
        lp = density_loss_adjoint(p, _run(s, Vp, Wp, nsteps, True)[0].rho, T.rho)[0]
        lm = density_loss_adjoint(p, _run(s, Vm, Wm, nsteps, True)[0].rho, T.rho)[0]
        fd = (lp - lm) / (2 * h)
        ad = sum(float(x @ y) for x, y in zip(g0.arrays() + [gB0.Bx_f, gB0.By_f], dU.arrays() + [dB.Bx_f, dB.By_f]))
        assert abs(ad - fd) <= 1e-6 * abs(fd), f"direction: {ad} vs {fd}"
    # eta step 1e-7: in the periodic case a branch of the map (limiter or
    # Riemann-solver region) lies within 1e-6 of eta, which a 1e-6 central
    # difference straddles; the loss's roundoff over 1e-7 stays below 1e-7
    de = 1e-7
    losses = []
    for e in (p.eta + de, p.eta - de):
        with AdjointSolver(replace(p, eta=e), checkpoint_every=2, max_steps=nsteps) as s2:
            s2.set_dts(dts)
            losses.append(density_loss_adjoint(p, _run(s2, U, B, nsteps, True)[0].rho, T.rho)[0])
    fd_eta = (losses[0] - losses[1]) / (2 * de)
    assert abs(geta - fd_eta) <= 1e-6 * abs(fd_eta), f"eta: {geta} vs {fd_eta}"
