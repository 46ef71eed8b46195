// 2D Euler + self-gravity with HLLC (euler2d_gravity_hllc.cpp, cited EH:<line>),
// templated on T; instantiated per precision in euler2d_f64.cu / euler2d_f32.cu.
//
// One RK stage is one kernel.  A CTA owns a TX x TY tile of cells, builds the
// primitives of a halo-2 region in shared memory (each from a floored copy of
// the conserved state, EH:420-425), computes the x and y faces of its cells
// with the reference's 4-point MUSCL-MC stencil and HLLC, and applies
//   stage 1:  U1 = floors(U + dt rhs(U))                      (EH:530-540)
//   stage 2:  U  = floors(0.5 U + 0.5 (U1 + dt rhs(U1)))       (EH:542-549)
// where rhs includes the gravity source with g from the potential of the
// stage input (EH:411, 516-523).  Stage 2 writes U in place (it reads U only
// at its own cell).  Same pitched layout as the 2D MHD solver.
#pragma once
#include "mhd2d_physics.cuh"

namespace ccb {

template <class T> struct EHConst {
    T gamma, gm1, floor_rho, floor_P;
    T dx, dy, two_dx, two_dy;
    int nx, ny, pitch;
    AxisMap ax, ay;     // boundary rule of the fluxes
    AxisMap pax, pay;   // the Poisson solve always wraps (EH:300-304)
    int gravity_on;
};

template <class T> struct EHFields { T* rho; T* mx; T* my; T* E; };
template <class T> struct EPrim { T r, u, v, P; };

// enforce_floors (EH:62-72)
template <class T>
__device__ __forceinline__ void eh_floors(const EHConst<T>& c, T& rho, T mx, T my, T& E) {
    rho = vmax(rho, c.floor_rho);
    const T ir = recip_if_fast(rho);
    const T u = div_or_mul(mx, rho, ir), v = div_or_mul(my, rho, ir);
    const T kin = T(0.5) * rho * (u * u + v * v);
    const T P = c.gm1 * (E - kin);
    if (P < c.floor_P) {
        const T eint = c.floor_P / c.gm1;
        E = kin + eint;
    }
}

// cons_to_prim_full / cons_to_prim (EH:74-100); *a = sqrt(gamma P / rho)
template <class T>
__device__ __forceinline__ EPrim<T> eh_prim(const EHConst<T>& c, T rho, T mx, T my, T E, T* a = nullptr) {
    const T r = vmax(rho, c.floor_rho);
    const T ir = recip_if_fast(r);
    const T u = div_or_mul(mx, r, ir), v = div_or_mul(my, r, ir);
    const T kin = T(0.5) * r * (u * u + v * v);
    T P = c.gm1 * (E - kin);
    if (P < c.floor_P) P = c.floor_P;
    if (a) *a = sqrt(c.gamma * P / r);
    EPrim<T> W;
    W.r = r; W.u = u; W.v = v; W.P = P;
    return W;
}

// HLLC (EH:125-219).  DIR 0: x faces (normal u), 1: y faces (normal v).
// Star energy uses P, not P* (EH:154, 202); SM = 0 when |den| <= 1e-14.
template <class T, int DIR>
__device__ __forceinline__ void eh_hllc(const EHConst<T>& c, const EPrim<T>& L, const EPrim<T>& R, T F[4]) {
    const T aL = sqrt(c.gamma * L.P / vmax(L.r, c.floor_rho));
    const T aR = sqrt(c.gamma * R.P / vmax(R.r, c.floor_rho));
    const T nL = DIR == 0 ? L.u : L.v, nR = DIR == 0 ? R.u : R.v;
    const T SL = vmin(nL - aL, nR - aR);
    const T SR = vmax(nL + aL, nR + aR);
    // prim_to_cons (EH:102-109)
    const T rL = vmax(L.r, c.floor_rho), rR = vmax(R.r, c.floor_rho);
    const T mLx = rL * L.u, mLy = rL * L.v, mRx = rR * R.u, mRy = rR * R.v;
    const T igm1 = recip_if_fast(c.gm1);
    const T EL = T(0.5) * rL * (L.u * L.u + L.v * L.v) + div_or_mul(L.P, c.gm1, igm1);
    const T ER = T(0.5) * rR * (R.u * R.u + R.v * R.v) + div_or_mul(R.P, c.gm1, igm1);
    const T num = (R.P - L.P) + rL * nL * (SL - nL) - rR * nR * (SR - nR);
    const T den = rL * (SL - nL) - rR * (SR - nR);
    const T SM = (fabs(den) > T(1e-14)) ? (num / den) : T(0.0);
    // euler_flux_x / euler_flux_y (EH:113-123) of the chosen side
    const bool upL = (T(0.0) <= SL), upR = !(T(0.0) <= SL) && (T(0.0) >= SR);
    const bool left = upL || (!upR && (T(0.0) < SM));
    // the chosen side's state and wave speed, by value (a reference chosen at
    // run time would put L and R in local memory), selected before the early
    // return (see ns_hllc in ns2d_kernels.cuh)
    EPrim<T> W;
    W.r = left ? L.r : R.r; W.u = left ? L.u : R.u; W.v = left ? L.v : R.v; W.P = left ? L.P : R.P;
    const T S = left ? SL : SR;
    const T Ef = div_or_mul(W.P, c.gm1, igm1) + T(0.5) * W.r * (W.u * W.u + W.v * W.v);
    if (DIR == 0) {
        F[0] = W.r * W.u; F[1] = W.r * W.u * W.u + W.P; F[2] = W.r * W.u * W.v; F[3] = (Ef + W.P) * W.u;
    } else {
        F[0] = W.r * W.v; F[1] = W.r * W.u * W.v; F[2] = W.r * W.v * W.v + W.P; F[3] = (Ef + W.P) * W.v;
    }
    if (upL || upR) return;
    // star state of the chosen side (EH:147-156, 195-204)
    const T r = left ? rL : rR, E = left ? EL : ER;
    const T mx = left ? mLx : mRx, my = left ? mLy : mRy;
    const T n = DIR == 0 ? W.u : W.v, t = DIR == 0 ? W.v : W.u;
    const T iSS = recip_if_fast(S - SM);
    const T rS = div_or_mul(r * (S - n), S - SM, iSS);
    const T mn = rS * SM, mt = rS * t;
    const T ES = div_or_mul((S - n) * E - W.P * n + W.P * SM, S - SM, iSS);
    const T mxS = DIR == 0 ? mn : mt, myS = DIR == 0 ? mt : mn;
    F[0] = F[0] + S * (rS - r);
    F[1] = F[1] + S * (mxS - mx);
    F[2] = F[2] + S * (myS - my);
    F[3] = F[3] + S * (ES - E);
}

// FP64 tiles are 31 cells wide (ROWW): a row of x faces is then 32 wide, and
// the y faces and cells are also mapped one row per warp (a lane per column,
// the last one idle), so no warp straddles two rows and every face loop is
// one round.  At 4096^2 that took the FP64 step from 4.16 to 3.81 ms; the same
// for FP32 (31 x 15 on 512 threads) made it slower (2.11 -> 2.39 ms: the
// FP32 stage is bound by the tile's loads, and its 10% more, smaller tiles
// cost more than the rounds and bank conflicts saved), so FP32 keeps 32 x 16.
template <class T> struct EHTile;
template <> struct EHTile<double> { static constexpr int TX = 31, TY = 8, NT = 288; };
template <> struct EHTile<float> { static constexpr int TX = 32, TY = 16, NT = 512; };

template <class T> struct EHGeom {
    static constexpr int TX = EHTile<T>::TX, TY = EHTile<T>::TY, HALO = 2;
    static constexpr int RX = TX + 2 * HALO, RY = TY + 2 * HALO, RR = RX * RY, NT = EHTile<T>::NT;
    static constexpr int NFX = (TX + 1) * TY, NGY = TX * (TY + 1);
    static constexpr bool ROWW = (TX == 31);
    static_assert(NT % 32 == 0 && (ROWW ? NT >= 32 * (TY + 1) : NT == TX * TY), "a thread per cell, whole warps");
    static constexpr size_t smem = sizeof(T) * (size_t)(4 * RR + 4 * NFX + 4 * NGY);
};

template <class T, bool STAGE2>
__global__ void __launch_bounds__(EHGeom<T>::NT, 2)
eh_stage_kernel(const EHConst<T> c, const EHFields<T> un, const EHFields<T> in, const EHFields<T> out,
                const T* __restrict__ phi, const T* __restrict__ gxa, const T* __restrict__ gya,
                const double* __restrict__ dtp, const int* __restrict__ active) {
    using G = EHGeom<T>;
    constexpr int TX = G::TX, TY = G::TY, HALO = G::HALO, RX = G::RX, RR = G::RR, NT = G::NT;
    constexpr int NFX = G::NFX, NGY = G::NGY;
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    T* s_r = sm; T* s_u = s_r + RR; T* s_v = s_u + RR; T* s_P = s_v + RR;
    T* fx = s_P + RR;        // 4 planes of NFX
    T* gy = fx + 4 * NFX;    // 4 planes of NGY
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int P = c.pitch;
    const T dt = (T)(*dtp);

    // primitives of floored copies over the halo-2 region (EH:420-425)
    for (int k = tid; k < RR; k += NT) {
        const int rx = k % RX, ry = k / RX;
        const size_t q = (size_t)c.ay.cell(j0 - HALO + ry) * P + c.ax.cell(i0 - HALO + rx);
        T rho = in.rho[q], mx = in.mx[q], my = in.my[q], E = in.E[q];
        eh_floors(c, rho, mx, my, E);
        const EPrim<T> W = eh_prim(c, rho, mx, my, E);
        s_r[k] = W.r; s_u[k] = W.u; s_v[k] = W.v; s_P[k] = W.P;
    }
    __syncthreads();

    // 4-point MUSCL-MC face states (EH:437-459): left = w0 + sL/2, right = wp - sR/2
    auto face = [&](int km, int k0, int kp, int kpp, EPrim<T>& L, EPrim<T>& R) {
        auto lr = [&](const T* s, T& l, T& r) {
            const T sL = mc_slope(s[km], s[k0], s[kp]);    // mc_limiter(w0 - wm, wp - w0)
            const T sR = mc_slope(s[k0], s[kp], s[kpp]);   // mc_limiter(wp - w0, wpp - wp)
            l = s[k0] + T(0.5) * sL;
            r = s[kp] - T(0.5) * sR;
        };
        lr(s_r, L.r, R.r); lr(s_u, L.u, R.u); lr(s_v, L.v, R.v); lr(s_P, L.P, R.P);
        L.r = vmax(L.r, c.floor_rho); R.r = vmax(R.r, c.floor_rho);
        L.P = vmax(L.P, c.floor_P); R.P = vmax(R.P, c.floor_P);
    };
    auto ridx = [&](int lx, int ly) { return (ly + HALO) * RX + (lx + HALO); };

    for (int k = tid; k < NFX; k += NT) {  // x faces i0..i0+TX of rows j0..j0+TY-1
        const int f = k % (TX + 1), r = k / (TX + 1);
        if (i0 + f > c.nx || j0 + r >= c.ny) continue;
        EPrim<T> L, R;
        face(ridx(f - 2, r), ridx(f - 1, r), ridx(f, r), ridx(f + 1, r), L, R);
        T F[4];
        eh_hllc<T, 0>(c, L, R, F);
        fx[k] = F[0]; fx[NFX + k] = F[1]; fx[2 * NFX + k] = F[2]; fx[3 * NFX + k] = F[3];
    }
    for (int kk = tid; kk < (G::ROWW ? 32 * (TY + 1) : NGY); kk += NT) {  // y faces j0..j0+TY of columns i0..i0+TX-1
        const int w = G::ROWW ? 32 : TX;
        const int col = kk % w, g = kk / w, k = g * TX + col;
        if (col >= TX || j0 + g > c.ny || i0 + col >= c.nx) continue;
        EPrim<T> L, R;
        face(ridx(col, g - 2), ridx(col, g - 1), ridx(col, g), ridx(col, g + 1), L, R);
        T F[4];
        eh_hllc<T, 1>(c, L, R, F);
        gy[k] = F[0]; gy[NGY + k] = F[1]; gy[2 * NGY + k] = F[2]; gy[3 * NGY + k] = F[3];
    }
    __syncthreads();

    const int tx = tid % (G::ROWW ? 32 : TX), ty = tid / (G::ROWW ? 32 : TX);
    const int gi = i0 + tx, gj = j0 + ty;
    if (tx >= TX || ty >= TY || gi >= c.nx || gj >= c.ny) return;
    const size_t q = (size_t)gj * P + gi;
    // rhs (EH:503-524): flux divergence, then the gravity source with the raw state
    const int kx = ty * (TX + 1) + tx, ky = ty * TX + tx;
    const T idx = recip_if_fast(c.dx), idy = recip_if_fast(c.dy);
    T d[4];
#pragma unroll
    for (int m = 0; m < 4; m++)
        d[m] = -div_or_mul(fx[m * NFX + kx + 1] - fx[m * NFX + kx], c.dx, idx) -
               div_or_mul(gy[m * NGY + ky + TX] - gy[m * NGY + ky], c.dy, idy);
    const T r0 = in.rho[q], mx0 = in.mx[q], my0 = in.my[q], E0 = in.E[q];
    if (c.gravity_on) {
        T gxq, gyq;
        if (gxa) {   // gravity given as arrays (enclosed-mass gravity)
            gxq = gxa[q];
            gyq = gya[q];
        } else {
            const int iE = c.pax.cell(gi + 1), iW = c.pax.cell(gi - 1);
            const int jN = c.pay.cell(gj + 1), jS = c.pay.cell(gj - 1);
            gxq = div_or_mul(-(phi[(size_t)gj * P + iE] - phi[(size_t)gj * P + iW]), c.two_dx, T(0.5) * idx);
            gyq = div_or_mul(-(phi[(size_t)jN * P + gi] - phi[(size_t)jS * P + gi]), c.two_dy, T(0.5) * idy);
        }
        const T rho = vmax(r0, c.floor_rho);
        const T ir = recip_if_fast(rho);
        const T u = div_or_mul(mx0, rho, ir), v = div_or_mul(my0, rho, ir);
        d[1] += rho * gxq;
        d[2] += rho * gyq;
        d[3] += rho * (u * gxq + v * gyq);
    }
    T rho, mx, my, E;
    if (!STAGE2) {
        rho = r0 + dt * d[0]; mx = mx0 + dt * d[1]; my = my0 + dt * d[2]; E = E0 + dt * d[3];
    } else {
        rho = T(0.5) * un.rho[q] + T(0.5) * (r0 + dt * d[0]);
        mx = T(0.5) * un.mx[q] + T(0.5) * (mx0 + dt * d[1]);
        my = T(0.5) * un.my[q] + T(0.5) * (my0 + dt * d[2]);
        E = T(0.5) * un.E[q] + T(0.5) * (E0 + dt * d[3]);
    }
    eh_floors(c, rho, mx, my, E);
    out.rho[q] = rho; out.mx[q] = mx; out.my[q] = my; out.E[q] = E;
}

// CFL speeds (EH:396-402) and the floored-density sum the Poisson mean needs
// (EH:309-317), FP64 block partials.
template <class T, int NT>
__global__ void __launch_bounds__(NT)
eh_speed_kernel(const EHConst<T> c, const EHFields<T> s, double* __restrict__ spd_part, double* __restrict__ rho_part) {
    __shared__ double sh[NT / 32];
    double smax = 0.0, rsum = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const int i = k % c.nx, j = k / c.nx;
        const size_t q = (size_t)j * c.pitch + i;
        T a;
        const EPrim<T> W = eh_prim(c, s.rho[q], s.mx[q], s.my[q], s.E[q], &a);
        const double sx = (double)(fabs(W.u) + a), sy = (double)(fabs(W.v) + a);
        if (sx > smax) smax = sx;   // std::max(maxs, x) never keeps a NaN
        if (sy > smax) smax = sy;
        rsum += (double)vmax(s.rho[q], c.floor_rho);
    }
    const double bm = block_max<NT>(smax, sh);
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) { spd_part[blockIdx.x] = bm; rho_part[blockIdx.x] = bs; }
}

template <class T, int NT>
__global__ void __launch_bounds__(NT)
eh_rho_sum_kernel(const EHConst<T> c, const T* __restrict__ rho, double* __restrict__ rho_part) {
    __shared__ double sh[NT / 32];
    double rsum = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT)
        rsum += (double)vmax(rho[(size_t)(k / c.nx) * c.pitch + (k % c.nx)], c.floor_rho);
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) rho_part[blockIdx.x] = bs;
}

// Snapshot fields of the reference main()'s store (EH:661-689): out[0..2] =
// rho, P, Mach per cell (3 planes of nx*ny doubles): floors on a copy of the
// cell, cons_to_prim_full, Mach = |v| / a (0 where a <= 0).
template <class T>
__global__ void eh_derived_kernel(const EHConst<T> c, const EHFields<T> s, double* __restrict__ out) {
    const size_t n = (size_t)c.nx * c.ny;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const size_t q = (k / c.nx) * c.pitch + (k % c.nx);
        T rho = s.rho[q], E = s.E[q];
        const T mx = s.mx[q], my = s.my[q];
        eh_floors(c, rho, mx, my, E);
        T a;
        const EPrim<T> W = eh_prim(c, rho, mx, my, E, &a);
        const T vmag = sqrt(W.u * W.u + W.v * W.v);
        out[k] = rho;
        out[n + k] = W.P;
        out[2 * n + k] = (a > T(0.0)) ? (vmag / a) : T(0.0);
    }
}

template <class T, int NT>
__global__ void __launch_bounds__(NT) eh_diag_kernel(const EHConst<T> c, const EHFields<T> s, double* __restrict__ part) {
    __shared__ double sh[NT / 32];
    double acc[4] = {0, 0, 0, 0}, nonf = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const size_t q = (size_t)(k / c.nx) * c.pitch + (k % c.nx);
        const double v[4] = {(double)s.rho[q], (double)s.mx[q], (double)s.my[q], (double)s.E[q]};
        for (int m = 0; m < 4; m++) {
            acc[m] += v[m];
            if (!isfinite(v[m])) nonf = 1.0;
        }
    }
    for (int m = 0; m < 4; m++) {
        const double b = block_sum<NT>(acc[m], sh);
        if (threadIdx.x == 0) part[m * gridDim.x + blockIdx.x] = b;
    }
    const double bn = block_max<NT>(nonf, sh);
    if (threadIdx.x == 0) part[4 * gridDim.x + blockIdx.x] = bn;
}

}  // namespace ccb
