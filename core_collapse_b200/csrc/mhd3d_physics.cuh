// Pointwise physics of the 3D resistive-MHD step (mhd3d_resistive_hlld_ct.cpp,
// cited M3:<line>): the hybrid cold + thermal EOS with bounce stiffening, as
// overloads on M3Const so that the shared HLLD template (mhd2d_physics.cuh)
// uses it.  Same evaluation order as the reference; the FP64 build is
// -fmad=false.
#pragma once
#include "mhd2d_physics.cuh"

namespace ccb {

template <class T> struct M3Const {
    // EOS (M3:43-53)
    T g1, g2, K1, K2, rn, gth, rb, gb, Kb;
    T g1m1, g2m1, gbm1, gthm1;   // gamma - 1 of each piece
    T e1n, e2n, pbb, ebb;         // K1 rn^(g1-1)/(g1-1), K2 rn^(g2-1)/(g2-1), rb^gb, rb^(gb-1): host std::pow
    int cold_off;                 // K1 == 0 and Kbounce == 0: the cold part is identically zero
    T floor_rho, floor_P, eta;
    T dx, dy, dz, inv_dx, inv_dy, inv_dz, two_dx, two_dy, two_dz;
    int nx, ny, nz;
    int P;                        // row pitch (elements)
    long long PS;                 // plane stride (elements)
    AxisMap ax, ay, az;
    int resistive;
    __host__ __device__ __forceinline__ size_t idx(int i, int j, int k) const {
        return (size_t)k * (size_t)PS + (size_t)j * (size_t)P + (size_t)i;
    }
};

template <class T> struct ColdEos { T P, e, g; };

// eos_cold (M3:118-144).  With K1 = Kbounce = 0 every cold term is 0 times a
// finite power, i.e. exactly 0, and the adiabatic index is gamma1, gamma2, or
// 0 above rho_bounce (0 / floor_P); the shortcut returns those bits directly.
template <class T>
__host__ __device__ __forceinline__ ColdEos<T> eos_cold(const M3Const<T>& c, T rho) {
    rho = vmax(rho, c.floor_rho);
    ColdEos<T> r;
    if (c.cold_off) {
        r.P = T(0.0); r.e = T(0.0);
        r.g = (rho < c.rn) ? c.g1
                           : ((rho >= c.rb) ? (c.g2 * (T(0.0) - T(0.0)) + c.gb * T(0.0)) / vmax(T(0.0), c.floor_P)
                                            : c.g2);
        return r;
    }
    if (rho < c.rn) {
        r.P = c.K1 * pow(rho, c.g1);
        r.e = c.K1 * pow(rho, c.g1m1) / c.g1m1;
        r.g = c.g1;
        return r;
    }
    T Pc = c.K2 * pow(rho, c.g2);
    T ec = c.e1n + (c.K2 * pow(rho, c.g2m1) / c.g2m1 - c.e2n);
    T gc = c.g2;
    if (rho >= c.rb) {
        const T pb = c.Kb * (pow(rho, c.gb) - c.pbb);
        const T eb = c.Kb * (pow(rho, c.gbm1) - c.ebb) / c.gbm1;
        Pc += pb;
        ec += eb;
        gc = (c.g2 * (Pc - pb) + c.gb * pb) / vmax(Pc, c.floor_P);
    }
    r.P = Pc; r.e = ec; r.g = gc;
    return r;
}

// pressure_from_rho_espec (M3:146-152)
template <class T>
__host__ __device__ __forceinline__ T eos_pressure(const M3Const<T>& c, T rho, T e_spec) {
    rho = vmax(rho, c.floor_rho);
    const ColdEos<T> cd = eos_cold(c, rho);
    const T eth = vmax(T(0.0), e_spec - cd.e);
    const T Pth = c.gthm1 * rho * eth;
    return vmax(cd.P + Pth, c.floor_P);
}

// total_energy_from_prim (M3:154-163)
template <class T>
__host__ __device__ __forceinline__ T energy(const M3Const<T>& c, const Prim<T>& W) {
    const T rho = vmax(W.r, c.floor_rho);
    const T kin = T(0.5) * rho * (W.u * W.u + W.v * W.v + W.w * W.w);
    const T mag = T(0.5) * (W.bx * W.bx + W.by * W.by + W.bz * W.bz);
    const ColdEos<T> cd = eos_cold(c, rho);
    const T Pth = vmax(T(0.0), W.P - cd.P);
    const T eth = (c.gth > T(1.0)) ? (Pth / (c.gthm1 * rho)) : T(0.0);
    const T eint = rho * (cd.e + eth);
    return kin + mag + eint;
}

// enforce_floors (M3:165-183): always re-projects E through the EOS
template <class T>
__host__ __device__ __forceinline__ void floors(const M3Const<T>& c, T& rho, T mx, T my, T mz, T& E, T Bx, T By, T Bz) {
    rho = vmax(rho, c.floor_rho);
    const T ir = recip_if_fast(rho);
    const T u = div_or_mul(mx, rho, ir), v = div_or_mul(my, rho, ir), w = div_or_mul(mz, rho, ir);
    const T kin = T(0.5) * rho * (u * u + v * v + w * w);
    const T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
    T eint = E - kin - mag;
    if (eint < T(0.0)) eint = T(0.0);
    const T es = div_or_mul(eint, rho, ir);
    T P = eos_pressure(c, rho, es);
    if (P < c.floor_P) P = c.floor_P;
    const ColdEos<T> cd = eos_cold(c, rho);
    const T Pth = vmax(T(0.0), P - cd.P);
    const T eth = (c.gth > T(1.0)) ? (Pth / (c.gthm1 * rho)) : T(0.0);
    const T en = rho * (cd.e + eth);
    E = kin + mag + en;
}

// cons_to_prim (M3:185-197)
template <class T>
__host__ __device__ __forceinline__ Prim<T> to_prim(const M3Const<T>& c, T rho, T mx, T my, T mz, T E, T Bx, T By, T Bz) {
    rho = vmax(rho, c.floor_rho);
    const T ir = recip_if_fast(rho);
    const T u = div_or_mul(mx, rho, ir), v = div_or_mul(my, rho, ir), w = div_or_mul(mz, rho, ir);
    const T kin = T(0.5) * rho * (u * u + v * v + w * w);
    const T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
    T eint = E - kin - mag;
    if (eint < T(0.0)) eint = T(0.0);
    const T es = div_or_mul(eint, rho, ir);
    T P = eos_pressure(c, rho, es);
    if (P < c.floor_P) P = c.floor_P;
    Prim<T> W;
    W.r = rho; W.u = u; W.v = v; W.w = w; W.P = P; W.bx = Bx; W.by = By; W.bz = Bz;
    return W;
}

// sound_speed2 (M3:206-212): (gamma_cold Pcold + gamma_th Pth) / rho, >= 0
template <class T>
__host__ __device__ __forceinline__ T sound_speed2(const M3Const<T>& c, const Prim<T>& W) {
    const T rhof = vmax(W.r, c.floor_rho);
    const ColdEos<T> cd = eos_cold(c, rhof);
    const T Pth = vmax(T(0.0), W.P - cd.P);
    const T num = cd.g * cd.P + c.gth * Pth;
    return vmax(T(0.0), num / rhof);
}

// fast magnetosonic speed with the hybrid sound speed (M3:206-248)
template <class T>
__device__ __forceinline__ T fast_speed(const M3Const<T>& c, const Prim<T>& W, T bn) {
    const T rhof = vmax(W.r, c.floor_rho);
    const ColdEos<T> cd = eos_cold(c, rhof);
    const T Pth = vmax(T(0.0), W.P - cd.P);
    const T num = cd.g * cd.P + c.gth * Pth;
    const T a2 = vmax(T(0.0), num / rhof);
    const T b2 = W.bx * W.bx + W.by * W.by + W.bz * W.bz;
    const T rho = vmax(W.r, tiny_pos<T>());
    const T ir = recip_if_fast(rho);
    const T vA2 = div_or_mul(b2, rho, ir);
    const T vn2 = div_or_mul(bn * bn, rho, ir);
    T disc = (a2 + vA2) * (a2 + vA2) - T(4.0) * a2 * vn2;
    disc = vmax(T(0.0), disc);
    const T cf2 = T(0.5) * ((a2 + vA2) + sqrt(disc));
    return sqrt(vmax(T(0.0), cf2));
}

}  // namespace ccb
