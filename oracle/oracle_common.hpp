// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// CPU restatement of the reference finite-volume step, used by tests/ and by
// bench.py's CPU-baseline leg as the checker.  This header holds the pieces
// shared by the 2D and 3D restatements: std::max/std::min/std::abs with the
// exact semantics the reference relies on, index wrapping, and the MC limiter.
//
// The restatement is templated on the arithmetic type T (double for parity,
// float for precision studies).  Every expression keeps the reference's
// evaluation order so that, compiled without FMA contraction
// (-ffp-contract=off), T=double reproduces the reference bit for bit.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <array>
#include <vector>

namespace cco {

// std::max(a,b) is (a<b)?b:a and std::min(a,b) is (b<a)?b:a; the NaN
// behaviour of these (first argument wins) matters in compute_dt.
template <class T> inline T vmax(T a, T b) { return (a < b) ? b : a; }
template <class T> inline T vmin(T a, T b) { return (b < a) ? b : a; }

// |a| and sqrt(a) found by argument-dependent lookup: std:: for double and
// float (unchanged results), the Dual overloads below for the tangent build.
template <class T> inline T oabs(T a) { using std::abs; return abs(a); }
template <class T> inline T osqrt(T a) { using std::sqrt; return sqrt(a); }

// Forward-mode dual number for the tangent-linear build of the restatement:
// v carries exactly the double operations of the value computation (so the
// value trajectory is bitwise the T = double one), d the directional
// derivative along the branch the value took.
struct Dual {
    double v, d;
    Dual(double x = 0.0) : v(x), d(0.0) {}
    Dual(double x, double dx) : v(x), d(dx) {}
};
inline Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
inline Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
inline Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
inline Dual operator/(Dual a, Dual b) {
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
inline Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
inline Dual operator+(Dual a) { return a; }
inline Dual& operator+=(Dual& a, Dual b) { return a = a + b; }
inline Dual& operator-=(Dual& a, Dual b) { return a = a - b; }
inline Dual& operator*=(Dual& a, Dual b) { return a = a * b; }
inline Dual& operator/=(Dual& a, Dual b) { return a = a / b; }
inline bool operator<(Dual a, Dual b) { return a.v < b.v; }
inline bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
inline bool operator>(Dual a, Dual b) { return a.v > b.v; }
inline bool operator>=(Dual a, Dual b) { return a.v >= b.v; }
inline bool operator==(Dual a, Dual b) { return a.v == b.v; }
inline bool operator!=(Dual a, Dual b) { return a.v != b.v; }
inline Dual abs(Dual a) { return a.v < 0.0 ? -a : a; }
inline Dual sqrt(Dual a) {
    const double r = std::sqrt(a.v);
    return Dual(r, r > 0.0 ? a.d / (2.0 * r) : 0.0);
}

inline int wrap_idx(int i, int n) { int r = i % n; return (r < 0) ? r + n : r; }
inline int clamp_idx(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }

// One axis of the grid: cell indices wrap modulo n (periodic) or clamp to
// [0,n-1]; face indices along the axis wrap modulo n+1 or clamp to [0,n]
// (mhd2d_resistive_hlld_ct_gravity.cpp:241-252).
struct Axis {
    int n;
    bool periodic;
    int cell(int i) const { return periodic ? wrap_idx(i, n) : clamp_idx(i, 0, n - 1); }
    int face(int i) const { return periodic ? wrap_idx(i, n + 1) : clamp_idx(i, 0, n); }
};

// minmod / MC limiter (M2:106-112, M3:106-112, EH:85-92).
template <class T> inline T minmod(T a, T b) {
    if (a * b <= T(0)) return T(0);
    return (oabs(a) < oabs(b)) ? a : b;
}
template <class T> inline T mc_slope(T dm, T dp) {
    return minmod(T(0.5) * (dm + dp), minmod(T(2.0) * dm, T(2.0) * dp));
}


template <class T> struct Prim8 { T r, u, v, w, P, bx, by, bz; };
template <class T> struct Flux7 { T f[7]; };  // rho, mx, my, mz, E, B_t1, B_t2

// x-normal ideal-MHD flux; the energy comes from the solver's EOS
// (M2:351-370 ideal gas, M3:396-413 hybrid EOS).
template <class T, class Phys> Flux7<T> ideal_flux_x(const Phys& ph, const Prim8<T>& W) {
    T rho = W.r, u = W.u, v = W.v, w = W.w, P = W.P, Bx = W.bx, By = W.by, Bz = W.bz;
    T B2 = Bx * Bx + By * By + Bz * Bz;
    T pt = P + T(0.5) * B2;
    T E = ph.energy(W);
    T vdotB = u * Bx + v * By + w * Bz;
    Flux7<T> F;
    F.f[0] = rho * u;
    F.f[1] = rho * u * u + pt - Bx * Bx;
    F.f[2] = rho * u * v - Bx * By;
    F.f[3] = rho * u * w - Bx * Bz;
    F.f[4] = (E + pt) * u - Bx * vdotB;
    F.f[5] = u * By - v * Bx;
    F.f[6] = u * Bz - w * Bx;
    return F;
}

// The reference HLLD (M2:372-530, identical in M3:415-568 up to the EOS):
// SM only for |denominator| > 1e-14, degenerate star states keep the outer B
// and v, HLL for |Bn| < 1e-12, double-star states jumped from the outer
// state with the outer speed, strict region tests.  Phys supplies
// energy(W) and fast(W, Bn*Bn).
template <class T, class Phys> Flux7<T> hlld_x_generic(const Phys& ph, Prim8<T> L, Prim8<T> R, T Bn) {
    L.bx = Bn; R.bx = Bn;
    Flux7<T> FL = ideal_flux_x(ph, L), FR = ideal_flux_x(ph, R);
    T cfL = ph.fast(L, L.bx * L.bx), cfR = ph.fast(R, R.bx * R.bx);
    T SL = vmin(L.u - cfL, R.u - cfR);
    T SR = vmax(L.u + cfL, R.u + cfR);
    if (T(0.0) <= SL) return FL;
    if (T(0.0) >= SR) return FR;

    std::array<T, 7> UL = {L.r, L.r * L.u, L.r * L.v, L.r * L.w, ph.energy(L), L.by, L.bz};
    std::array<T, 7> UR = {R.r, R.r * R.u, R.r * R.v, R.r * R.w, ph.energy(R), R.by, R.bz};
    T ptL = L.P + T(0.5) * (L.bx * L.bx + L.by * L.by + L.bz * L.bz);
    T ptR = R.P + T(0.5) * (R.bx * R.bx + R.by * R.by + R.bz * R.bz);

    T den = L.r * (SL - L.u) - R.r * (SR - R.u);
    T SM = T(0.0);
    if (oabs(den) > T(1e-14)) SM = (ptR - ptL + L.r * L.u * (SL - L.u) - R.r * R.u * (SR - R.u)) / den;

    T rLs = L.r * (SL - L.u) / (SL - SM);
    T rRs = R.r * (SR - R.u) / (SR - SM);
    T pts = ptL + L.r * (SL - L.u) * (SM - L.u);
    T sL = SL - L.u, sR = SR - R.u;
    T dL = L.r * sL * (SL - SM) - Bn * Bn;
    T dR = R.r * sR * (SR - SM) - Bn * Bn;

    T ByLs = L.by, BzLs = L.bz, ByRs = R.by, BzRs = R.bz;
    T vLs = L.v, wLs = L.w, vRs = R.v, wRs = R.w;
    if (oabs(dL) > T(1e-14)) {
        ByLs = L.by * (L.r * sL * (SL - L.u) - Bn * Bn) / dL;
        BzLs = L.bz * (L.r * sL * (SL - L.u) - Bn * Bn) / dL;
        vLs = L.v - Bn * (ByLs - L.by) / (L.r * (SL - L.u) * (SL - SM));
        wLs = L.w - Bn * (BzLs - L.bz) / (L.r * (SL - L.u) * (SL - SM));
    }
    if (oabs(dR) > T(1e-14)) {
        ByRs = R.by * (R.r * sR * (SR - R.u) - Bn * Bn) / dR;
        BzRs = R.bz * (R.r * sR * (SR - R.u) - Bn * Bn) / dR;
        vRs = R.v - Bn * (ByRs - R.by) / (R.r * (SR - R.u) * (SR - SM));
        wRs = R.w - Bn * (BzRs - R.bz) / (R.r * (SR - R.u) * (SR - SM));
    }
    T sqL = osqrt(vmax(rLs, T(1e-300)));
    T sqR = osqrt(vmax(rRs, T(1e-300)));
    T SLL = SM - oabs(Bn) / sqL;
    T SRR = SM + oabs(Bn) / sqR;

    if (oabs(Bn) < T(1e-12)) {  // HLL fallback (M2:449-467)
        T inv = T(1.0) / (SR - SL);
        Flux7<T> F;
        for (int k = 0; k < 7; k++) F.f[k] = (SR * FL.f[k] - SL * FR.f[k] + SL * SR * (UR[k] - UL[k])) * inv;
        return F;
    }
    T sgn = (Bn >= T(0.0)) ? T(1.0) : T(-1.0);
    T d2 = sqL + sqR;
    T vss = (sqL * vLs + sqR * vRs + (ByRs - ByLs) * sgn) / d2;
    T wss = (sqL * wLs + sqR * wRs + (BzRs - BzLs) * sgn) / d2;
    T Byss = (sqL * ByRs + sqR * ByLs + sqL * sqR * (vRs - vLs) * sgn) / d2;
    T Bzss = (sqL * BzRs + sqR * BzLs + sqL * sqR * (wRs - wLs) * sgn) / d2;

    // star state relative to the outer state W (M2:486-505)
    auto ustar = [&](const Prim8<T>& W, T S, T rs, T vs, T ws, T Bys, T Bzs) {
        T EW = ph.energy(W);
        T vBs = SM * Bn + vs * Bys + ws * Bzs;
        T vBw = W.u * W.bx + W.v * W.by + W.w * W.bz;
        T ptW = W.P + T(0.5) * (W.bx * W.bx + W.by * W.by + W.bz * W.bz);
        T E = ((S - W.u) * EW - (ptW * W.u - Bn * vBw) + (pts * SM - Bn * vBs)) / (S - SM);
        return std::array<T, 7>{rs, rs * SM, rs * vs, rs * ws, E, Bys, Bzs};
    };
    auto jump = [&](const std::array<T, 7>& Us, const std::array<T, 7>& U0, const Flux7<T>& F0, T S) {
        Flux7<T> F;
        for (int k = 0; k < 7; k++) F.f[k] = F0.f[k] + S * (Us[k] - U0[k]);
        return F;
    };
    if (T(0.0) < SLL) return jump(ustar(L, SL, rLs, vLs, wLs, ByLs, BzLs), UL, FL, SL);
    if (T(0.0) < SM) return jump(ustar(L, SL, rLs, vss, wss, Byss, Bzss), UL, FL, SL);
    if (T(0.0) < SRR) return jump(ustar(R, SR, rRs, vss, wss, Byss, Bzss), UR, FR, SR);
    return jump(ustar(R, SR, rRs, vRs, wRs, ByRs, BzRs), UR, FR, SR);
}

}  // namespace cco
