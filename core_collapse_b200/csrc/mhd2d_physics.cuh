// Pointwise physics of the 2D resistive-MHD step, device side, templated on
// the arithmetic type T (double: parity path, float: bulk path).
//
// Every expression keeps the evaluation order of mhd2d_resistive_hlld_ct_gravity.cpp
// (cited M2:<line>); the double instantiation is compiled with -fmad=false so
// that it rounds exactly like the reference's x86-64 build.
#pragma once
#include "cc_device.cuh"

namespace ccb {

template <class T> struct M2Const {
    T gamma, gm1;          // gamma, gamma-1
    T floor_rho, floor_P;
    T eta;
    T dx, dy;
    T inv_dx, inv_dy;      // 1/dx, 1/dy        (M2:750)
    T idx2, idy2;          // 1/dx^2, 1/dy^2    (M2:668)
    T two_dx, two_dy;      // 2*dx, 2*dy        (M2:232, 646)
    int nx, ny, pitch;
    AxisMap ax, ay;
    int gravity_on;
    int resistive;         // eta > 0
};

template <class T> struct Prim { T r, u, v, w, P, bx, by, bz; };
template <class T> struct Flux { T f0, f1, f2, f3, f4, f5, f6; };  // rho,mx,my,mz,E,Bt1,Bt2

// One of two states by value, component-wise (a reference chosen at run time
// would force both states into local memory).
template <class T>
__host__ __device__ __forceinline__ Prim<T> prim_select(bool left, const Prim<T>& L, const Prim<T>& R) {
    Prim<T> W;
    W.r = left ? L.r : R.r; W.u = left ? L.u : R.u; W.v = left ? L.v : R.v; W.w = left ? L.w : R.w;
    W.P = left ? L.P : R.P; W.bx = left ? L.bx : R.bx; W.by = left ? L.by : R.by; W.bz = left ? L.bz : R.bz;
    return W;
}

// The FP32 bulk path is issue-bound and each of its divisions is several
// instructions, so where one denominator serves several quotients it takes
// one reciprocal and multiplies (a rounding change of an ulp); FP64 keeps the
// reference's divisions operation for operation.
template <class T> __host__ __device__ constexpr bool fast_recip() { return sizeof(T) == 4; }

// 1/b on the fast-reciprocal path, else 0 (never read there): the FP64 build
// forms no division that it does not use
template <class T> __host__ __device__ __forceinline__ T recip_if_fast(T b) {
    if constexpr (fast_recip<T>()) return T(1.0) / b;
    else return T(0.0);
}

// a / b; a * ib on the fast-reciprocal path (ib = 1/b, precomputed)
template <class T> __host__ __device__ __forceinline__ T div_or_mul(T a, T b, T ib) {
    if constexpr (fast_recip<T>()) return a * ib;
    else return a / b;
}

// enforce_floors (M2:114-124)
template <class T>
__host__ __device__ __forceinline__ void floors(const M2Const<T>& c, T& rho, T mx, T my, T mz, T& E, T Bx, T By, T Bz) {
    rho = vmax(rho, c.floor_rho);
    T u, v, w;
    if constexpr (fast_recip<T>()) {
        const T ir = T(1.0) / rho;
        u = mx * ir; v = my * ir; w = mz * ir;
    } else {
        u = mx / rho; v = my / rho; w = mz / rho;
    }
    T kin = T(0.5) * rho * (u * u + v * v + w * w);
    T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
    T P = c.gm1 * (E - kin - mag);
    if (P < c.floor_P) {
        T eint = c.floor_P / c.gm1;
        E = kin + mag + eint;
    }
}

// cons_to_prim (M2:126-135)
template <class T>
__host__ __device__ __forceinline__ Prim<T> to_prim(const M2Const<T>& c, T rho, T mx, T my, T mz, T E, T Bx, T By, T Bz) {
    rho = vmax(rho, c.floor_rho);
    T u, v, w;
    if constexpr (fast_recip<T>()) {
        const T ir = T(1.0) / rho;
        u = mx * ir; v = my * ir; w = mz * ir;
    } else {
        u = mx / rho; v = my / rho; w = mz / rho;
    }
    T kin = T(0.5) * rho * (u * u + v * v + w * w);
    T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
    T P = c.gm1 * (E - kin - mag);
    if (P < c.floor_P) P = c.floor_P;
    Prim<T> W;
    W.r = rho; W.u = u; W.v = v; W.w = w; W.P = P; W.bx = Bx; W.by = By; W.bz = Bz;
    return W;
}

// total energy of a primitive state, ideal gas (M2:357, 397, 482, 495)
template <class T>
__host__ __device__ __forceinline__ T energy(const M2Const<T>& c, const Prim<T>& W) {
    T B2 = W.bx * W.bx + W.by * W.by + W.bz * W.bz;
    T eint;
    if constexpr (fast_recip<T>()) eint = W.P * (T(1.0) / c.gm1);   // 1/gm1 shared by every call in a face
    else eint = W.P / c.gm1;
    return eint + T(0.5) * W.r * (W.u * W.u + W.v * W.v + W.w * W.w) + T(0.5) * B2;
}

// fast magnetosonic speed with normal component bn (M2:148-174)
template <class T>
__host__ __device__ __forceinline__ T fast_speed(const M2Const<T>& c, const Prim<T>& W, T bn) {
    T b2 = W.bx * W.bx + W.by * W.by + W.bz * W.bz;
    T a2, vA2, vn2;
    if constexpr (fast_recip<T>()) {
        // every caller passes a floored density (face states, cons_to_prim), so
        // the two floors of the reference's expression select the same value and
        // one reciprocal serves the three quotients
        const T ir = T(1.0) / vmax(W.r, c.floor_rho);
        a2 = c.gamma * W.P * ir;
        vA2 = b2 * ir;
        vn2 = (bn * bn) * ir;
    } else {
        a2 = c.gamma * W.P / vmax(W.r, c.floor_rho);
        const T rho = vmax(W.r, T(1e-300));
        vA2 = b2 / rho;
        vn2 = (bn * bn) / rho;
    }
    T disc = (a2 + vA2) * (a2 + vA2) - T(4.0) * a2 * vn2;
    disc = vmax(T(0.0), disc);
    T cf2 = T(0.5) * ((a2 + vA2) + sqrt(disc));
    return sqrt(vmax(T(0.0), cf2));
}

// x-normal ideal flux (M2:351-370; M3:396-413 with the hybrid-EOS energy).
// Cst is the solver's constant block: energy(c, W) and fast_speed(c, W, bn)
// are overloaded on it.
template <class T, class Cst>
__host__ __device__ __forceinline__ Flux<T> ideal_flux(const Cst& c, const Prim<T>& W) {
    T rho = W.r, u = W.u, v = W.v, w = W.w, P = W.P, Bx = W.bx, By = W.by, Bz = W.bz;
    T B2 = Bx * Bx + By * By + Bz * Bz;
    T pt = P + T(0.5) * B2;
    T E = energy(c, W);
    T vdotB = u * Bx + v * By + w * Bz;
    Flux<T> F;
    F.f0 = rho * u;
    F.f1 = rho * u * u + pt - Bx * Bx;
    F.f2 = rho * u * v - Bx * By;
    F.f3 = rho * u * w - Bx * Bz;
    F.f4 = (E + pt) * u - Bx * vdotB;
    F.f5 = u * By - v * Bx;
    F.f6 = u * Bz - w * Bx;
    return F;
}

// ideal_flux of a state whose total energy E and total pressure pt are known
// (the same expressions as ideal_flux forms them, so the same values)
template <class T>
__host__ __device__ __forceinline__ Flux<T> ideal_flux_ep(const Prim<T>& W, T E, T pt) {
    T rho = W.r, u = W.u, v = W.v, w = W.w, Bx = W.bx, By = W.by, Bz = W.bz;
    T vdotB = u * Bx + v * By + w * Bz;
    Flux<T> F;
    F.f0 = rho * u;
    F.f1 = rho * u * u + pt - Bx * Bx;
    F.f2 = rho * u * v - Bx * By;
    F.f3 = rho * u * w - Bx * Bz;
    F.f4 = (E + pt) * u - Bx * vdotB;
    F.f5 = u * By - v * Bx;
    F.f6 = u * Bz - w * Bx;
    return F;
}

// HLLD (M2:372-530), the reference's own star / double-star construction:
// degenerate guards at 1e-14, HLL fallback for |Bn| < 1e-12, double-star
// fluxes jumped from the outer state with the outer speed.
template <class T, class Cst>
__host__ __device__ __forceinline__ Flux<T> hlld_x(const Cst& c, Prim<T> L, Prim<T> R, T Bn) {
    L.bx = Bn; R.bx = Bn;
    const T cfL = fast_speed(c, L, Bn), cfR = fast_speed(c, R, Bn);
    const T SL = vmin(L.u - cfL, R.u - cfR);
    const T SR = vmax(L.u + cfL, R.u + cfR);
    if (T(0.0) <= SL) return ideal_flux(c, L);
    if (T(0.0) >= SR) return ideal_flux(c, R);

    const T EL = energy(c, L), ER = energy(c, R);
    const T ptL = L.P + T(0.5) * (L.bx * L.bx + L.by * L.by + L.bz * L.bz);
    const T ptR = R.P + T(0.5) * (R.bx * R.bx + R.by * R.by + R.bz * R.bz);

    if (fabs(Bn) < T(1e-12)) {  // HLL (M2:449-467)
        const Flux<T> FL = ideal_flux(c, L), FR = ideal_flux(c, R);
        const T inv = T(1.0) / (SR - SL);
        const T s2 = SL * SR;
        Flux<T> F;
        F.f0 = (SR * FL.f0 - SL * FR.f0 + s2 * (R.r - L.r)) * inv;
        F.f1 = (SR * FL.f1 - SL * FR.f1 + s2 * (R.r * R.u - L.r * L.u)) * inv;
        F.f2 = (SR * FL.f2 - SL * FR.f2 + s2 * (R.r * R.v - L.r * L.v)) * inv;
        F.f3 = (SR * FL.f3 - SL * FR.f3 + s2 * (R.r * R.w - L.r * L.w)) * inv;
        F.f4 = (SR * FL.f4 - SL * FR.f4 + s2 * (ER - EL)) * inv;
        F.f5 = (SR * FL.f5 - SL * FR.f5 + s2 * (R.by - L.by)) * inv;
        F.f6 = (SR * FL.f6 - SL * FR.f6 + s2 * (R.bz - L.bz)) * inv;
        return F;
    }

    const T den = L.r * (SL - L.u) - R.r * (SR - R.u);
    T SM = T(0.0);
    if (fabs(den) > T(1e-14)) SM = (ptR - ptL + L.r * L.u * (SL - L.u) - R.r * R.u * (SR - R.u)) / den;

    const T rLs = L.r * (SL - L.u) / (SL - SM);
    const T rRs = R.r * (SR - R.u) / (SR - SM);
    const T pts = ptL + L.r * (SL - L.u) * (SM - L.u);
    const T sL = SL - L.u, sR = SR - R.u;
    const T bn2 = Bn * Bn;
    const T dL = L.r * sL * (SL - SM) - bn2;
    const T dR = R.r * sR * (SR - SM) - bn2;

    T ByLs = L.by, BzLs = L.bz, ByRs = R.by, BzRs = R.bz;
    T vLs = L.v, wLs = L.w, vRs = R.v, wRs = R.w;
    if (fabs(dL) > T(1e-14)) {
        const T num = L.r * sL * (SL - L.u) - bn2;
        const T dd = L.r * (SL - L.u) * (SL - SM);
        if constexpr (fast_recip<T>()) {
            const T q = num / dL, bq = Bn / dd;
            ByLs = L.by * q;
            BzLs = L.bz * q;
            vLs = L.v - (ByLs - L.by) * bq;
            wLs = L.w - (BzLs - L.bz) * bq;
        } else {
            ByLs = L.by * num / dL;
            BzLs = L.bz * num / dL;
            vLs = L.v - Bn * (ByLs - L.by) / dd;
            wLs = L.w - Bn * (BzLs - L.bz) / dd;
        }
    }
    if (fabs(dR) > T(1e-14)) {
        const T num = R.r * sR * (SR - R.u) - bn2;
        const T dd = R.r * (SR - R.u) * (SR - SM);
        if constexpr (fast_recip<T>()) {
            const T q = num / dR, bq = Bn / dd;
            ByRs = R.by * q;
            BzRs = R.bz * q;
            vRs = R.v - (ByRs - R.by) * bq;
            wRs = R.w - (BzRs - R.bz) * bq;
        } else {
            ByRs = R.by * num / dR;
            BzRs = R.bz * num / dR;
            vRs = R.v - Bn * (ByRs - R.by) / dd;
            wRs = R.w - Bn * (BzRs - R.bz) / dd;
        }
    }
    T sqL, sqR, SLL, SRR;
    if constexpr (fast_recip<T>()) {
        // one reciprocal square root each: sqrt(r) = r / sqrt(r), |Bn| / sqrt(r)
        const T rl = vmax(rLs, T(1e-30)), rr = vmax(rRs, T(1e-30));
        const T iqL = rsqrt(rl), iqR = rsqrt(rr);
        sqL = rl * iqL;
        sqR = rr * iqR;
        // explicit fused multiply-adds: the same rounding in every kernel that inlines this
        SLL = __fmaf_rn(-fabs(Bn), iqL, SM);
        SRR = __fmaf_rn(fabs(Bn), iqR, SM);
    } else {
        sqL = sqrt(vmax(rLs, T(1e-300)));
        sqR = sqrt(vmax(rRs, T(1e-300)));
        SLL = SM - fabs(Bn) / sqL;
        SRR = SM + fabs(Bn) / sqR;
    }

    // pick the region first, then build only the state it needs
    const bool left = (T(0.0) < SM);
    const bool outer = left ? (T(0.0) < SLL) : !(T(0.0) < SRR);
    const Prim<T> W = prim_select(left, L, R);
    const T S = left ? SL : SR;
    const T EW = left ? EL : ER;
    const T ptW = left ? ptL : ptR;
    T rs = left ? rLs : rRs, vs, ws, Bys, Bzs;
    if (outer) {
        vs = left ? vLs : vRs; ws = left ? wLs : wRs;
        Bys = left ? ByLs : ByRs; Bzs = left ? BzLs : BzRs;
    } else {
        const T sgn = (Bn >= T(0.0)) ? T(1.0) : T(-1.0);
        const T d2 = sqL + sqR;
        if constexpr (fast_recip<T>()) {
            const T id2 = T(1.0) / d2;
            vs = (sqL * vLs + sqR * vRs + (ByRs - ByLs) * sgn) * id2;
            ws = (sqL * wLs + sqR * wRs + (BzRs - BzLs) * sgn) * id2;
            Bys = (sqL * ByRs + sqR * ByLs + sqL * sqR * (vRs - vLs) * sgn) * id2;
            Bzs = (sqL * BzRs + sqR * BzLs + sqL * sqR * (wRs - wLs) * sgn) * id2;
        } else {
            vs = (sqL * vLs + sqR * vRs + (ByRs - ByLs) * sgn) / d2;
            ws = (sqL * wLs + sqR * wRs + (BzRs - BzLs) * sgn) / d2;
            Bys = (sqL * ByRs + sqR * ByLs + sqL * sqR * (vRs - vLs) * sgn) / d2;
            Bzs = (sqL * BzRs + sqR * BzLs + sqL * sqR * (wRs - wLs) * sgn) / d2;
        }
    }
    // U_star (M2:486-505) and the jump F_W + S (U* - U_W) (M2:507-519)
    const T vBs = SM * Bn + vs * Bys + ws * Bzs;
    const T vBw = W.u * W.bx + W.v * W.by + W.w * W.bz;
    const T Es = ((S - W.u) * EW - (ptW * W.u - Bn * vBw) + (pts * SM - Bn * vBs)) / (S - SM);
    // FP64: the flux from the known energy and total pressure (the same values);
    // FP32 forms them again, which keeps its rounding the same in every kernel
    // that inlines this (the batched tile shapes give bit-identical results)
    Flux<T> F;
    if constexpr (fast_recip<T>()) F = ideal_flux(c, W);
    else F = ideal_flux_ep(W, EW, ptW);
    F.f0 = F.f0 + S * (rs - W.r);
    F.f1 = F.f1 + S * (rs * SM - W.r * W.u);
    F.f2 = F.f2 + S * (rs * vs - W.r * W.v);
    F.f3 = F.f3 + S * (rs * ws - W.r * W.w);
    F.f4 = F.f4 + S * (Es - EW);
    F.f5 = F.f5 + S * (Bys - W.by);
    F.f6 = F.f6 + S * (Bzs - W.bz);
    return F;
}

// y-normal HLLD through the (u,v)/(Bx,By) swap (M2:540-561).  Returns
// f1 = flux of mx, f2 = flux of my, f5 = flux of Bx (= Ez at the y face), f6 = flux of Bz.
template <class T, class Cst>
__host__ __device__ __forceinline__ Flux<T> hlld_y(const Cst& c, const Prim<T>& L, const Prim<T>& R, T Bn) {
    Prim<T> aL, aR;
    aL.r = L.r; aL.u = L.v; aL.v = L.u; aL.w = L.w; aL.P = L.P; aL.bx = Bn; aL.by = L.bx; aL.bz = L.bz;
    aR.r = R.r; aR.u = R.v; aR.v = R.u; aR.w = R.w; aR.P = R.P; aR.bx = Bn; aR.by = R.bx; aR.bz = R.bz;
    Flux<T> F = hlld_x(c, aL, aR, Bn);
    const T t = F.f1; F.f1 = F.f2; F.f2 = t;
    return F;
}

// z-normal HLLD through the cyclic (w,u,v)/(Bz,Bx,By) map (M3:604-622).
// Returns f1 = F(mx), f2 = F(my), f3 = F(mz), f5 = F(Bx), f6 = F(By).
template <class T, class Cst>
__host__ __device__ __forceinline__ Flux<T> hlld_z(const Cst& c, const Prim<T>& L, const Prim<T>& R, T Bn) {
    Prim<T> aL, aR;
    aL.r = L.r; aL.u = L.w; aL.v = L.u; aL.w = L.v; aL.P = L.P; aL.bx = Bn; aL.by = L.bx; aL.bz = L.by;
    aR.r = R.r; aR.u = R.w; aR.v = R.u; aR.w = R.v; aR.P = R.P; aR.bx = Bn; aR.by = R.bx; aR.bz = R.by;
    Flux<T> F = hlld_x(c, aL, aR, Bn);
    const T fmx = F.f2, fmy = F.f3, fmz = F.f1;
    F.f1 = fmx; F.f2 = fmy; F.f3 = fmz;
    return F;
}

// MC-limited slope (M2:106-112, 295)
template <class T> __host__ __device__ __forceinline__ T minmod(T a, T b) {
    if (a * b <= T(0.0)) return T(0.0);
    return (fabs(a) < fabs(b)) ? a : b;
}
template <class T> __host__ __device__ __forceinline__ T mc_slope(T wm, T wc, T wp) {
    const T dm = wc - wm, dp = wp - wc;
    return minmod(T(0.5) * (dm + dp), minmod(T(2.0) * dm, T(2.0) * dp));
}

}  // namespace ccb
