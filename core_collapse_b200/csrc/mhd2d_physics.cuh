// Pointwise physics of the 2D resistive-MHD step, device side, templated on
// the arithmetic type T (double: parity path, float: bulk path).
//
// Every expression keeps the evaluation order of mhd2d_resistive_hlld_ct_gravity.cpp
// (cited M2:<line>); the double instantiation is compiled with -fmad=false so
// that it rounds exactly like the reference's x86-64 build.
#pragma once
#include <type_traits>

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
        const T rho = vmax(W.r, tiny_pos<T>());
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
__host__ __device__ __forceinline__ Flux<T> hlld_x_scalar(const Cst& c, Prim<T> L, Prim<T> R, T Bn) {
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
        sqL = sqrt(vmax(rLs, tiny_pos<T>()));
        sqR = sqrt(vmax(rRs, tiny_pos<T>()));
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

// ---------------------------------------------------------------------------
// HLLD of the 2D FP32 path on packed FP32 pairs.  sm_100 executes add, mul
// and fma on a float2 (.f32x2) as one instruction; HLLD forms the same
// quantities for its left and right states (fast speeds, energies, total
// pressures, star states, Alfven speeds), so the FP32 path keeps each such
// pair in one float2, .x the left state and .y the right, and spends one
// issue slot where the scalar code spends two.  Each lane rounds like the
// scalar FP32 code with its multiply-adds contracted (divisions, square roots
// and comparisons stay scalar).  The region logic and the flux of the chosen
// state follow hlld_x_scalar line for line; its max / min are fmaxf / fminf
// (one instruction where (a < b) ? b : a takes a compare and a select; the
// same value for every operand that is not NaN).
// ---------------------------------------------------------------------------
struct Prim2 { float2 r, u, v, w, P, bx, by, bz; };   // .x left state, .y right state

__device__ __forceinline__ float2 pk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 pbc(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b as fma(b, -1, a): one rounding, the exact difference rounded
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, pbc(-1.0f), a); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ Prim<float> lane_x(const Prim2& S) {
    return Prim<float>{S.r.x, S.u.x, S.v.x, S.w.x, S.P.x, S.bx.x, S.by.x, S.bz.x};
}
__device__ __forceinline__ Prim<float> lane_y(const Prim2& S) {
    return Prim<float>{S.r.y, S.u.y, S.v.y, S.w.y, S.P.y, S.bx.y, S.by.y, S.bz.y};
}

__device__ __forceinline__ Flux<float> hlld_x2(const M2Const<float>& c, Prim2 S, const float Bn) {
    const float2 bn = pbc(Bn);
    S.bx = bn;
    // fast_speed of both states (M2:148-174)
    const float2 bn2p = pmul(bn, bn);
    const float2 b2 = pfma(S.bz, S.bz, pfma(S.by, S.by, bn2p));
    const float2 ir = pk(1.0f / fmaxf(S.r.x, c.floor_rho), 1.0f / fmaxf(S.r.y, c.floor_rho));
    const float2 a2 = pmul(pmul(pbc(c.gamma), S.P), ir);
    const float2 vA2 = pmul(b2, ir);
    const float2 vn2 = pmul(bn2p, ir);
    const float2 sa = padd(a2, vA2);
    const float2 disc = pfma(sa, sa, pmul(pmul(pbc(-4.0f), a2), vn2));
    const float2 sd = pk(sqrtf(fmaxf(0.0f, disc.x)), sqrtf(fmaxf(0.0f, disc.y)));
    const float2 cf2 = pmul(pbc(0.5f), padd(sa, sd));
    const float2 cf = pk(sqrtf(fmaxf(0.0f, cf2.x)), sqrtf(fmaxf(0.0f, cf2.y)));
    const float2 um = psub(S.u, cf), up = padd(S.u, cf);
    const float SL = fminf(um.x, um.y);
    const float SR = fmaxf(up.x, up.y);
    if (0.0f <= SL) return ideal_flux(c, lane_x(S));
    if (0.0f >= SR) return ideal_flux(c, lane_y(S));

    // energies and total pressures (M2:357, 482, 495)
    const float2 ksum = pfma(S.w, S.w, pfma(S.v, S.v, pmul(S.u, S.u)));
    const float2 eint = pmul(S.P, pbc(1.0f / c.gm1));
    const float2 E = pfma(pbc(0.5f), b2, pfma(pmul(pbc(0.5f), S.r), ksum, eint));
    const float2 pt = pfma(pbc(0.5f), b2, S.P);

    if (fabsf(Bn) < 1e-12f) {  // HLL (M2:449-467)
        const Prim<float> L = lane_x(S), R = lane_y(S);
        const Flux<float> FL = ideal_flux(c, L), FR = ideal_flux(c, R);
        const float inv = 1.0f / (SR - SL);
        const float s2 = SL * SR;
        Flux<float> F;
        F.f0 = (SR * FL.f0 - SL * FR.f0 + s2 * (R.r - L.r)) * inv;
        F.f1 = (SR * FL.f1 - SL * FR.f1 + s2 * (R.r * R.u - L.r * L.u)) * inv;
        F.f2 = (SR * FL.f2 - SL * FR.f2 + s2 * (R.r * R.v - L.r * L.v)) * inv;
        F.f3 = (SR * FL.f3 - SL * FR.f3 + s2 * (R.r * R.w - L.r * L.w)) * inv;
        F.f4 = (SR * FL.f4 - SL * FR.f4 + s2 * (E.y - E.x)) * inv;
        F.f5 = (SR * FL.f5 - SL * FR.f5 + s2 * (R.by - L.by)) * inv;
        F.f6 = (SR * FL.f6 - SL * FR.f6 + s2 * (R.bz - L.bz)) * inv;
        return F;
    }

    // contact speed and star states (M2:470-505)
    const float2 SLR = pk(SL, SR);
    const float2 sLR = psub(SLR, S.u);          // SL - uL, SR - uR
    const float2 rsd = pmul(S.r, sLR);          // rho (S - u) of each side
    const float den = rsd.x - rsd.y;
    float SM = 0.0f;
    if (fabsf(den) > 1e-14f) {
        const float2 m = pmul(pmul(S.r, S.u), sLR);
        SM = (pt.y - pt.x + m.x - m.y) / den;
    }
    const float2 SmM = psub(SLR, pbc(SM));     // S - SM of each side
    const float2 rst = pk(rsd.x / SmM.x, rsd.y / SmM.y);
    const float pts = pt.x + rsd.x * (SM - S.u.x);
    const float bn2 = Bn * Bn;
    const float2 dLR = pfma(rsd, SmM, pbc(-bn2));
    const float2 num = pfma(rsd, sLR, pbc(-bn2));
    const float2 dd = pmul(rsd, SmM);
    const float2 q = pk(num.x / dLR.x, num.y / dLR.y);
    const float2 bq = pk(Bn / dd.x, Bn / dd.y);
    float2 Bys2 = pmul(S.by, q), Bzs2 = pmul(S.bz, q);
    float2 vs2 = pfma(psub(S.by, Bys2), bq, S.v);
    float2 ws2 = pfma(psub(S.bz, Bzs2), bq, S.w);
    if (!(fabsf(dLR.x) > 1e-14f)) { Bys2.x = S.by.x; Bzs2.x = S.bz.x; vs2.x = S.v.x; ws2.x = S.w.x; }
    if (!(fabsf(dLR.y) > 1e-14f)) { Bys2.y = S.by.y; Bzs2.y = S.bz.y; vs2.y = S.v.y; ws2.y = S.w.y; }
    const float2 rl = pk(fmaxf(rst.x, 1e-30f), fmaxf(rst.y, 1e-30f));
    const float2 iq = pk(rsqrtf(rl.x), rsqrtf(rl.y));
    const float2 sq = pmul(rl, iq);                                  // sqrt(rho*) of each side
    const float2 SAl = pfma(pk(-fabsf(Bn), fabsf(Bn)), iq, pbc(SM));  // SL*, SR*

    // the region, then only the state it needs (as hlld_x_scalar)
    const bool left = (0.0f < SM);
    const bool outer = left ? (0.0f < SAl.x) : !(0.0f < SAl.y);
    const Prim<float> W = prim_select(left, lane_x(S), lane_y(S));
    const float Sw = left ? SL : SR;
    const float EW = left ? E.x : E.y;
    const float ptW = left ? pt.x : pt.y;
    const float rs = left ? rst.x : rst.y;
    float vs, ws, Bys, Bzs;
    if (outer) {
        vs = left ? vs2.x : vs2.y; ws = left ? ws2.x : ws2.y;
        Bys = left ? Bys2.x : Bys2.y; Bzs = left ? Bzs2.x : Bzs2.y;
    } else {
        const float sgn = (Bn >= 0.0f) ? 1.0f : -1.0f;
        const float id2 = 1.0f / (sq.x + sq.y);
        vs = (sq.x * vs2.x + sq.y * vs2.y + (Bys2.y - Bys2.x) * sgn) * id2;
        ws = (sq.x * ws2.x + sq.y * ws2.y + (Bzs2.y - Bzs2.x) * sgn) * id2;
        Bys = (sq.x * Bys2.y + sq.y * Bys2.x + sq.x * sq.y * (vs2.y - vs2.x) * sgn) * id2;
        Bzs = (sq.x * Bzs2.y + sq.y * Bzs2.x + sq.x * sq.y * (ws2.y - ws2.x) * sgn) * id2;
    }
    const float vBs = SM * Bn + vs * Bys + ws * Bzs;
    const float vBw = W.u * W.bx + W.v * W.by + W.w * W.bz;
    const float Es = ((Sw - W.u) * EW - (ptW * W.u - Bn * vBw) + (pts * SM - Bn * vBs)) / (Sw - SM);
    Flux<float> F = ideal_flux(c, W);
    F.f0 = F.f0 + Sw * (rs - W.r);
    F.f1 = F.f1 + Sw * (rs * SM - W.r * W.u);
    F.f2 = F.f2 + Sw * (rs * vs - W.r * W.v);
    F.f3 = F.f3 + Sw * (rs * ws - W.r * W.w);
    F.f4 = F.f4 + Sw * (Es - EW);
    F.f5 = F.f5 + Sw * (Bys - W.by);
    F.f6 = F.f6 + Sw * (Bzs - W.bz);
    return F;
}

// HLLD of a face: the packed form on the 2D FP32 device path, else the scalar one
template <class T, class Cst>
__host__ __device__ __forceinline__ Flux<T> hlld_x(const Cst& c, const Prim<T>& L, const Prim<T>& R, T Bn) {
#if defined(__CUDA_ARCH__)
    if constexpr (std::is_same<Cst, M2Const<float>>::value) {
        const Prim2 S{pk(L.r, R.r), pk(L.u, R.u), pk(L.v, R.v), pk(L.w, R.w),
                      pk(L.P, R.P), pk(L.bx, R.bx), pk(L.by, R.by), pk(L.bz, R.bz)};
        return hlld_x2(c, S, Bn);
    } else {
        return hlld_x_scalar(c, L, R, Bn);
    }
#else
    return hlld_x_scalar(c, L, R, Bn);
#endif
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
    if constexpr (sizeof(T) == 4) {
        // FP32: the same limiter in fewer compare / select instructions (the
        // stage kernel's ALU pipe is its busiest): 0 when dm dp <= 0, else the
        // smallest of |dm + dp| / 2, 2 |dm|, 2 |dp|, with the sign of dm, which
        // is the value the two minmods select (ties have equal values)
        const T sc = T(0.5) * (dm + dp);
        const T m = fminf(fabsf(sc), fminf(fabsf(T(2.0) * dm), fabsf(T(2.0) * dp)));
        return (dm * dp <= T(0.0)) ? T(0.0) : copysignf(m, dm);
    } else {
        return minmod(T(0.5) * (dm + dp), minmod(T(2.0) * dm, T(2.0) * dp));
    }
}

}  // namespace ccb
