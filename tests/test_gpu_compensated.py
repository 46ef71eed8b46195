"""The compensated (Kahan-style) FP32 state update (cc_mhd2d_params.compensated).

A compensated handle keeps every state plane as an FP32 value plus its FP32
rounding residual and adds each stage increment and the RK average with an
error-free sum (the conserved update of mhd2d_resistive_hlld_ct_gravity.cpp:
750-779, the CT update :807-830 and the RK average :848-868).  Checked here:
the upload/download split carries an FP64 state to ~2^-48 relative; on the
FFT-gravity workload the compensated FP32 run is closer to the FP64 oracle
than the plain FP32 run in L1; FP64 handles and the ensemble reject the
option."""
import numpy as np
import pytest

import oracle_lib as O
from core_collapse_b200 import _lib as L
from core_collapse_b200.batch import BatchSolver
from core_collapse_b200.mhd2d import CcError, Mhd2dSolver, Params, ic_orszag_tang

pytestmark = pytest.mark.gpu

FIELDS = ["rho", "mx", "my", "mz", "E", "Bz", "Bx_f", "By_f"]


def _params(n, precision="fp32", compensated=True, **kw):
    d = dict(Nx=n, Ny=n, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=True, periodic_y=True, gamma=5.0 / 3.0,
             G=1.0, eta=1e-3, cfl=0.4, gravity_on=True, poisson="fft", precision=precision,
             compensated=compensated, t_end=1e30)
    d.update(kw)
    return Params(**d)


def _l1(a, b):
    den = float(np.sum(np.abs(b)))
    return float(np.sum(np.abs(a - b))) / den if den > 0 else float(np.max(np.abs(a - b)))


def test_upload_download_keeps_fp64_digits():
    p = _params(64)
    U, B = ic_orszag_tang(p, core_amp=4.0, core_width=0.1)
    with Mhd2dSolver(p) as s:
        s.upload(U, B)
        got = O.state_list(*s.download())
    for k, (a, b) in enumerate(zip(got, O.state_list(U, B))):
        assert O.rel_linf(a, b) <= 2.0 ** -46, FIELDS[k]


def test_compensated_closer_to_fp64_oracle():
    n, steps = 256, 40
    p64 = _params(n, "fp64", False)
    U, B = ic_orszag_tang(p64, core_amp=4.0, core_width=0.1)
    want, t_want = O.m2_main_loop_oracle(p64.to_c(), O.state_list(U, B), steps, mode=2)
    errs = {}
    for comp in (False, True):
        p = _params(n, "fp32", comp, t_end=t_want)
        with Mhd2dSolver(p) as s:
            s.upload(U, B)
            t = s.advance(steps + 4, 0.0)
            got = O.state_list(*s.download())
            d = s.diagnostics()
        assert abs(t - t_want) <= 1e-12 * t_want
        assert d["nonfinite"] == 0
        errs[comp] = {FIELDS[k]: _l1(a, b) for k, (a, b) in enumerate(zip(got, want)) if np.any(b != 0)}
    print("L1 vs FP64 oracle, plain / compensated:",
          {k: f"{errs[False][k]:.2e} / {errs[True][k]:.2e}" for k in errs[False]})
    assert max(errs[True].values()) < max(errs[False].values())


def test_compensated_rejected_where_unsupported():
    with pytest.raises(CcError) as e:
        Mhd2dSolver(_params(32, "fp64", True))
    assert e.value.code == L.CC_ERR_UNSUPPORTED
    p = Params(Nx=32, Ny=32, x0=-1.0, x1=1.0, y0=-1.0, y1=1.0, periodic_x=False, periodic_y=False, G=1.0,
               gravity_on=True, poisson="direct", precision="fp32", compensated=True)
    with pytest.raises(CcError) as e:
        BatchSolver([p])
    assert e.value.code == L.CC_ERR_UNSUPPORTED
