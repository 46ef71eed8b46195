"""Local vector-Jacobian products of the 2D MHD step's pointwise physics
(core_collapse_b200/csrc/mhd2d_adjoint.cuh) against central finite
differences, on the CPU through a host-compiled harness of the same headers.

Each check draws inputs in the regimes that select each branch (supersonic
left/right, HLL at Bn = 0, HLLD left/right x outer/inner regions, floored
density and pressure, every limiter choice) and compares lambda^T J e_i with
(lambda.F(x + h e_i) - lambda.F(x - h e_i)) / 2h for every input i.  Inputs
whose two-step finite differences disagree (a branch boundary within h) are
skipped; at least 90% of the components must be checkable."""
import ctypes as C
import sys
import zlib
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).resolve().parent / "native"))
import build as native_build  # noqa: E402

_DP = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def H():
    L = C.CDLL(str(native_build.build("adj_local")))
    for n in ("fwd_hlld", "vjp_hlld", "fwd_to_prim", "vjp_to_prim", "fwd_floors", "vjp_floors", "vjp_mc",
              "fwd_joule", "vjp_joule"):
        getattr(L, n).restype = None
    L.fwd_mc.restype = C.c_double
    L.fwd_mc.argtypes = [C.c_double] * 3
    L.vjp_mc.argtypes = [C.c_double] * 4 + [_DP]
    return L


def p(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a.ctypes.data_as(_DP)


# gamma, floor_rho, floor_P, eta, dx, dy
K = np.array([5.0 / 3.0, 1e-10, 1e-10, 1e-3, 2.0 / 64, 2.0 / 48])


def fd_check(f, x, lam, grad, rel=1e-6, min_ok=0.9, skip=()):
    """f: x -> output vector.  Compare grad[i] with the FD of lam.f along e_i
    (indices in `skip` sit on a branch boundary by construction)."""
    ok = len(skip)
    scale = np.max(np.abs(grad)) + 1e-30
    for i in range(len(x)):
        if i in skip:
            continue
        h = 1e-6 * max(1.0, abs(x[i]))
        d = []
        for hh in (h, h / 4):
            xp, xm = x.copy(), x.copy()
            xp[i] += hh
            xm[i] -= hh
            d.append((lam @ f(xp) - lam @ f(xm)) / (2 * hh))
        if abs(d[0] - d[1]) > 1e-5 * (abs(d[1]) + scale):
            continue   # branch boundary within h
        ok += 1
        assert abs(grad[i] - d[1]) <= rel * scale + 1e-6 * abs(d[1]), f"component {i}: vjp {grad[i]} fd {d[1]}"
    assert ok >= min_ok * len(x)


def _hlld_case(rng, regime):
    L = np.array([1.0, 0.2, -0.3, 0.1, 1.0, 0.0, 0.5, -0.2]) * (1 + 0.3 * rng.random(8))
    R = np.array([0.7, -0.1, 0.2, -0.2, 0.6, 0.0, -0.3, 0.4]) * (1 + 0.3 * rng.random(8))
    Bn = 0.4 * (1 + 0.2 * rng.random())
    if regime == "sup_left":
        L[1] = R[1] = 8.0
    elif regime == "sup_right":
        L[1] = R[1] = -8.0
    elif regime == "hll":
        Bn = 0.0
    elif regime == "left_outer":
        L[1], R[1], Bn = 1.0, 0.8, 0.05
    elif regime == "right_outer":
        L[1], R[1], Bn = -0.8, -1.0, 0.05
    elif regime == "inner":
        L[1], R[1], Bn = 0.02, -0.01, 1.5
    elif regime == "inner_negbn":
        L[1], R[1], Bn = -0.03, 0.02, -1.2
    return L, R, Bn


@pytest.mark.parametrize("dir_", [0, 1])
@pytest.mark.parametrize("regime", ["sup_left", "sup_right", "hll", "left_outer", "right_outer", "inner",
                                    "inner_negbn", "random"])
def test_hlld_vjp(H, dir_, regime):
    rng = np.random.default_rng(zlib.crc32(f"{dir_}{regime}".encode()))
    for _ in range(4):
        L, R, Bn = _hlld_case(rng, regime)
        if dir_ == 1:   # y faces: normal velocity is v, normal B is by
            L[[1, 2]] = L[[2, 1]]
            R[[1, 2]] = R[[2, 1]]
        lam = rng.normal(size=7)
        x = np.concatenate([L, R, [Bn]])
        nidx = 5 if dir_ == 0 else 6   # the forward overwrites the normal B of L and R with Bn

        def f(z):
            F = np.zeros(7)
            H.fwd_hlld(p(K), dir_, p(z[:8]), p(z[8:16]), C.c_double(z[16]), p(F))
            return F

        lL, lR, lBn = np.zeros(8), np.zeros(8), C.c_double()
        H.vjp_hlld(p(K), dir_, p(L), p(R), C.c_double(Bn), p(lam), p(lL), p(lR), C.byref(lBn))
        g = np.concatenate([lL, lR, [lBn.value]])
        assert g[nidx] == 0.0 and g[8 + nidx] == 0.0
        # at Bn = 0 any finite step in Bn leaves the HLL branch (|Bn| < 1e-12, M2:449)
        fd_check(f, x, lam, g, skip=(16,) if regime == "hll" else ())


@pytest.mark.parametrize("regime", ["plain", "rho_floor", "p_floor"])
def test_to_prim_and_floors_vjp(H, regime):
    rng = np.random.default_rng(7)
    k = K.copy()
    for _ in range(6):
        U = np.array([1.3, 0.4, -0.2, 0.3, 2.5, 0.2, 0.3, -0.4]) * (1 + 0.2 * rng.random(8))
        if regime == "rho_floor":
            k[1] = 2.0     # density floor above rho
        if regime == "p_floor":
            U[4] = 0.3     # E below kinetic + magnetic: pressure floored
            k[2] = 0.05
        lam = rng.normal(size=8)

        def fp(z):
            W = np.zeros(8)
            H.fwd_to_prim(p(k), p(z), p(W))
            return W

        g = np.zeros(8)
        H.vjp_to_prim(p(k), p(U), p(lam), p(g))
        fd_check(fp, U, lam, g)

        def ff(z):
            o = np.zeros(8)
            H.fwd_floors(p(k), p(z), p(o))
            return o

        g2 = np.zeros(8)
        H.vjp_floors(p(k), p(U), p(lam), p(g2))
        fd_check(ff, U, lam, g2)


def test_mc_slope_vjp_all_branches(H):
    rng = np.random.default_rng(3)
    seen = set()
    for _ in range(400):
        a = rng.normal(size=3)
        ls = rng.normal()
        out = np.zeros(3)
        H.vjp_mc(a[0], a[1], a[2], ls, p(out))
        dm, dp = a[1] - a[0], a[2] - a[1]
        s = H.fwd_mc(*a)
        seen.add("zero" if s == 0 else ("central" if abs(s - 0.5 * (dm + dp)) < 1e-15 else "limited"))
        fd_check(lambda z: np.array([H.fwd_mc(*z)]), a, np.array([ls]), out, min_ok=0.6)
    assert seen == {"zero", "central", "limited"}


@pytest.mark.parametrize("floored", [False, True])
def test_joule_vjp(H, floored):
    rng = np.random.default_rng(11)
    k = K.copy()
    k[3] = 3e-3
    for _ in range(5):
        x = np.concatenate([[1.1, 0.3, -0.2, 0.1, 2.0 if not floored else 0.2, 0.4, 0.3, -0.2],
                            rng.normal(scale=0.5, size=8)])
        if floored:
            k[2] = 0.2
        lam = rng.normal(size=6)

        def f(z):
            o = np.zeros(6)
            H.fwd_joule(p(k), C.c_double(0.01), p(z), p(o))
            return o

        g = np.zeros(17)
        H.vjp_joule(p(k), C.c_double(0.01), p(x), p(lam), p(g))
        fd_check(f, x, lam, g[:16])

        def feta(e):
            kk = k.copy()
            kk[3] = e[0]
            o = np.zeros(6)
            H.fwd_joule(p(kk), C.c_double(0.01), p(x), p(o))
            return o

        fd_check(feta, np.array([k[3]]), lam, g[16:17])
