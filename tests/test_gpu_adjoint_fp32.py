"""The adjoint of the FP32 forward (cc_adjoint_create with precision CC_FP32):
an FP32 forward run recorded and checkpointed, reversed by the same kernels
instantiated in FP32 (eta's adjoint summed in FP64).

A finite difference of an FP32 map measures its rounding, not its derivative,
so the FP32 gradients are checked against the FP64 adjoint of the same run
(itself checked against finite differences to 1e-6 in test_gpu_adjoint.py):
the density-misfit gradient with respect to the initial state and eta, with
the FP64 run replaying the FP32 run's recorded dt so both differentiate the
same discrete map.  Agreement is bounded by FP32 rounding along the
trajectory: relative to the largest entry, <= 2e-3 for the density gradient
and the eta derivative, <= 2e-2 for every field."""
import numpy as np
import pytest

from cases_adjoint import make_case_adj
from core_collapse_b200.adjoint import AdjointSolver, density_loss_adjoint

pytestmark = pytest.mark.gpu

TOL = 2e-3


@pytest.mark.parametrize("periodic,grav", [(False, True), (True, False)])
def test_fp32_adjoint_matches_fp64_adjoint(periodic, grav):
    from dataclasses import replace
    p, U, B = make_case_adj(periodic, grav, nx=48, ny=40)
    _, T, _ = make_case_adj(periodic, grav, nx=48, ny=40, seed=9)
    nsteps = 12
    grads = {}
    dts = None
    for prec in ("fp32", "fp64"):
        with AdjointSolver(replace(p, precision=prec), checkpoint_every=4, max_steps=nsteps) as s:
            s.upload(U, B)
            if dts is None:
                s.forward(nsteps)
                dts = s.dts()
            else:
                s.set_dts(dts)
                s.forward(nsteps, replay=True)
            UT, _ = s.download()
            loss, lamU, lamB = density_loss_adjoint(p, UT.rho, T.rho)
            g, gB, geta = s.vjp(lamU, lamB)
            grads[prec] = (loss, g, gB, geta, UT)
    l32, g32, gB32, e32, U32 = grads["fp32"]
    l64, g64, gB64, e64, U64 = grads["fp64"]
    traj = np.max(np.abs(U32.rho - U64.rho)) / np.max(np.abs(U64.rho))
    names = ["rho", "mx", "my", "mz", "E", "Bz"]
    errs = {}
    for k, (a, b) in enumerate(zip(g32.arrays(), g64.arrays())):
        scale = float(np.max(np.abs(b)))
        errs[names[k]] = float(np.max(np.abs(a - b))) / scale if scale > 0 else float(np.max(np.abs(a)))
    for name, a, b in (("Bx_f", gB32.Bx_f, gB64.Bx_f), ("By_f", gB32.By_f, gB64.By_f)):
        errs[name] = float(np.max(np.abs(a - b))) / max(float(np.max(np.abs(b))), 1e-300)
    print(f"FP32 trajectory vs FP64 {traj:.1e}; loss {l32:.6e} / {l64:.6e}; gradient errors "
          + ", ".join(f"{k} {v:.1e}" for k, v in errs.items()) + f"; eta {e32:.6e} / {e64:.6e}")
    assert traj <= 1e-4
    assert abs(l32 - l64) <= 1e-3 * abs(l64)
    assert errs["rho"] <= TOL
    assert max(errs.values()) <= 10 * TOL
    assert abs(e32 - e64) <= TOL * abs(e64)
