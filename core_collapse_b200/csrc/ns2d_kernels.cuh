// 2D compressible Navier-Stokes (explicit viscosity) + FFT self-gravity
// (navier_stokes_2d_hllc_poisson.cpp, cited NS:<line>), templated on T;
// instantiated per precision in ns2d_f64.cu (-fmad=false, the parity path)
// and ns2d_f32.cu.  Periodic in both directions.
//
// One Heun (SSP-RK2) stage is one kernel.  A CTA owns a TX x TY tile of cells
// and keeps in shared memory
//   * the primitives of the stage input over a halo-2 region (cons_to_prim, NS:119-132),
//   * the centred velocity gradients over a halo-1 region (NS:402-424),
//   * the x and y face fluxes of its cells: first-order HLLC of the two
//     adjacent cells (NS:212-282, 387-398) plus the viscous stress flux built
//     from face averages of the gradients (NS:426-480),
// and applies
//   stage 1:  k1 = rhs(U);  U1 = U + dt k1,            rho floored   (NS:762-771)
//   stage 2:  k2 = rhs(U1); U  = U + dt/2 (k1 + k2),   rho floored   (NS:773-781)
// with rhs = -div F + gravity source, g = -grad phi by centred differences of
// the potential of the stage input (NS:330-360, 500-513).  Stage 1 stores k1;
// stage 2 reads U and k1 only at its own cell and writes U in place.
#pragma once
#include "cc_device.cuh"

namespace ccb {

template <class T> struct NSConst {
    T gamma, gm1, floor_rho, floor_P;
    T mu;
    T idx1, idy1;   // 1/dx, 1/dy             (NS:485-486)
    T idx2, idy2;   // 1/(2 dx), 1/(2 dy)     (NS:340-341, 403-404)
    int nx, ny, pitch;
    int viscous;    // viscosity_on && mu > 0 (NS:400)
    int gravity_on;
};

template <class T> struct NSFields { T* d; T* mx; T* my; T* E; };
template <class T> struct NSPrim { T d, u, v, P; };

// cons_to_prim (NS:119-132)
template <class T>
__device__ __forceinline__ NSPrim<T> ns_prim(const NSConst<T>& c, T d, T mx, T my, T E) {
    NSPrim<T> W;
    W.d = vmax(d, c.floor_rho);
    if constexpr (sizeof(T) == 4) {   // FP32: one reciprocal (an ulp of rounding)
        const T id = T(1.0) / W.d;
        W.u = mx * id;
        W.v = my * id;
    } else {
        W.u = mx / W.d;
        W.v = my / W.d;
    }
    const T ke = T(0.5) * W.d * (W.u * W.u + W.v * W.v);
    const T eint = E - ke;
    const T P = c.gm1 * eint;
    W.P = vmax(P, c.floor_P);
    return W;
}

// sound_speed (NS:147-149)
template <class T>
__device__ __forceinline__ T ns_sound(const NSConst<T>& c, const NSPrim<T>& W) {
    return sqrt(c.gamma * W.P / vmax(W.d, c.floor_rho));
}

// hllc_x (NS:212-269) on (n, t) = (normal, tangential) velocity components;
// F = {mass, normal momentum, tangential momentum, energy}.  hllc_y (NS:271-282)
// is the same call with u and v exchanged and the momentum fluxes exchanged
// back.  Only the star state of the upwind side is formed (the reference
// forms both and returns one).
template <class T>
__device__ __forceinline__ void ns_hllc(const NSConst<T>& c, T dL, T nL, T tL, T pL, T dR, T nR, T tR, T pR,
                                        T F[4]) {
    const T aL = sqrt(c.gamma * pL / vmax(dL, c.floor_rho));
    const T aR = sqrt(c.gamma * pR / vmax(dR, c.floor_rho));
    // FP32 (issue-bound): 1/gm1 and 1/(S - SM) each formed once
    constexpr bool F32 = sizeof(T) == 4;
    const T igm1 = recip_if_fast(c.gm1);
    const T EL = (F32 ? pL * igm1 : pL / c.gm1) + T(0.5) * dL * (nL * nL + tL * tL);
    const T ER = (F32 ? pR * igm1 : pR / c.gm1) + T(0.5) * dR * (nR * nR + tR * tR);
    const T SL = vmin(nL - aL, nR - aR);
    const T SR = vmax(nL + aL, nR + aR);
    const T num = (pR - pL) + dL * nL * (SL - nL) - dR * nR * (SR - nR);
    const T den = dL * (SL - nL) - dR * (SR - nR);
    const T SM = (fabs(den) > T(0.0)) ? (num / den) : T(0.0);
    const bool upL = (T(0.0) <= SL), upR = !upL && (T(0.0) >= SR);
    const bool left = upL || (!upR && (T(0.0) < SM));
    // The chosen side's state and wave speed, by value (a run-time reference
    // would go to local memory), selected together in one branch: with nvcc
    // 12.9 for sm_100a, S selected on its own after the early return below
    // came out as the other side's speed for some faces (a unit probe of one
    // face reproduced it; the parity tests cover it).
    T d, n, t, p, E, S;
    if (left) { d = dL; n = nL; t = tL; p = pL; E = EL; S = SL; }
    else { d = dR; n = nR; t = tR; p = pR; E = ER; S = SR; }
    // flux_x_from_prim (NS:198-210)
    const T Ef = (F32 ? p * igm1 : p / c.gm1) + T(0.5) * d * (n * n + t * t);
    F[0] = d * n;
    F[1] = d * n * n + p;
    F[2] = d * n * t;
    F[3] = (Ef + p) * n;
    if (upL || upR) return;
    // Ustar (NS:235-249): star energy with the star pressure
    const T iSS = recip_if_fast(S - SM);
    const T fac = F32 ? d * (S - n) * iSS : d * (S - n) / (S - SM);
    const T pstar = p + d * (S - n) * (SM - n);
    const T Es = F32 ? ((S - n) * E - p * n + pstar * SM) * iSS : ((S - n) * E - p * n + pstar * SM) / (S - SM);
    F[0] = F[0] + S * (fac - d);
    F[1] = F[1] + S * (fac * SM - d * n);
    F[2] = F[2] + S * (fac * t - d * t);
    F[3] = F[3] + S * (Es - E);
}

// Tile TX x TY on NT threads, MINB CTAs per SM.  NT covers the larger face
// count ((TX+1) TY or TX (TY+1)) so that each face loop is one round; the
// extra threads idle in the update.
template <class T> struct NSTile;
template <> struct NSTile<double> { static constexpr int TX = 32, TY = 8, NT = 288, MINB = 2; };
template <> struct NSTile<float> { static constexpr int TX = 32, TY = 16, NT = 544, MINB = 3; };

template <class T> struct NSGeom {
    static constexpr int TX = NSTile<T>::TX, TY = NSTile<T>::TY, NT = NSTile<T>::NT, MINB = NSTile<T>::MINB;
    static constexpr int RX = TX + 4, RY = TY + 4, RR = RX * RY;   // primitives, halo 2
    static constexpr int GX = TX + 2, GY = TY + 2, GR = GX * GY;   // gradients, halo 1
    static constexpr int NFX = (TX + 1) * TY, NGY = TX * (TY + 1), NC = TX * TY;
    static_assert(NT >= NFX && NT >= NGY && NT % 32 == 0, "one round per face loop");
    static constexpr size_t smem = sizeof(T) * (size_t)(4 * RR + 4 * GR + 4 * NFX + 4 * NGY);
};

template <class T, bool STAGE2>
__global__ void __launch_bounds__(NSGeom<T>::NT, NSGeom<T>::MINB)
ns_stage_kernel(const NSConst<T> c, const NSFields<T> un, const NSFields<T> in, const NSFields<T> k1,
                const NSFields<T> out, const T* __restrict__ phi, const double* __restrict__ dtp,
                const int* __restrict__ active) {
    using G = NSGeom<T>;
    constexpr int TX = G::TX, TY = G::TY, RX = G::RX, RR = G::RR, GX = G::GX, GR = G::GR, NT = G::NT;
    constexpr int NFX = G::NFX, NGY = G::NGY;
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* sm = reinterpret_cast<T*>(smem_raw);
    T* s_d = sm; T* s_u = s_d + RR; T* s_v = s_u + RR; T* s_P = s_v + RR;
    T* g_ux = s_P + RR; T* g_uy = g_ux + GR; T* g_vx = g_uy + GR; T* g_vy = g_vx + GR;
    T* fx = g_vy + GR;       // 4 planes of NFX
    T* fy = fx + 4 * NFX;    // 4 planes of NGY
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * TX, j0 = blockIdx.y * TY;
    const int P = c.pitch;

    // primitives of the stage input over the halo-2 region (NS:372-377)
    for (int k = tid; k < RR; k += NT) {
        const int rx = k % RX, ry = k / RX;
        const size_t q = (size_t)wrap_idx(j0 - 2 + ry, c.ny) * P + wrap_idx(i0 - 2 + rx, c.nx);
        const NSPrim<T> W = ns_prim(c, in.d[q], in.mx[q], in.my[q], in.E[q]);
        s_d[k] = W.d; s_u[k] = W.u; s_v[k] = W.v; s_P[k] = W.P;
    }
    __syncthreads();
    auto r_at = [&](int lx, int ly) { return (ly + 2) * RX + (lx + 2); };   // tile coords -> primitive slot
    auto g_at = [&](int lx, int ly) { return (ly + 1) * GX + (lx + 1); };   // tile coords -> gradient slot

    if (c.viscous) {   // cell-centred velocity gradients (NS:402-424)
        for (int k = tid; k < GR; k += NT) {
            const int lx = k % GX - 1, ly = k / GX - 1;
            const int e = r_at(lx + 1, ly), w = r_at(lx - 1, ly), n = r_at(lx, ly + 1), s = r_at(lx, ly - 1);
            g_ux[k] = (s_u[e] - s_u[w]) * c.idx2;
            g_vx[k] = (s_v[e] - s_v[w]) * c.idx2;
            g_uy[k] = (s_u[n] - s_u[s]) * c.idy2;
            g_vy[k] = (s_v[n] - s_v[s]) * c.idy2;
        }
        __syncthreads();
    }

    // x faces: face f of row r lies between tile cells f-1 and f (Fx[i] of NS:387-392 with i = i0+f-1)
    for (int k = tid; k < NFX; k += NT) {
        const int f = k % (TX + 1), r = k / (TX + 1);
        const int L = r_at(f - 1, r), R = r_at(f, r);
        T F[4];
        ns_hllc(c, s_d[L], s_u[L], s_v[L], s_P[L], s_d[R], s_u[R], s_v[R], s_P[R], F);
        if (c.viscous) {   // NS:426-452
            const int gL = g_at(f - 1, r), gR = g_at(f, r);
            const T dudx = T(0.5) * (g_ux[gL] + g_ux[gR]);
            const T dudy = T(0.5) * (g_uy[gL] + g_uy[gR]);
            const T dvdx = T(0.5) * (g_vx[gL] + g_vx[gR]);
            const T dvdy = T(0.5) * (g_vy[gL] + g_vy[gR]);
            const T divv = dudx + dvdy;
            const T tau_xx = c.mu * (T(2.0) * dudx - (T(2.0) / T(3.0)) * divv);
            const T tau_xy = c.mu * (dudy + dvdx);
            const T uf = T(0.5) * (s_u[L] + s_u[R]);
            const T vf = T(0.5) * (s_v[L] + s_v[R]);
            F[1] += -tau_xx;
            F[2] += -tau_xy;
            F[3] += -(uf * tau_xx + vf * tau_xy);
        }
        fx[k] = F[0]; fx[NFX + k] = F[1]; fx[2 * NFX + k] = F[2]; fx[3 * NFX + k] = F[3];
    }
    // y faces: face g of column col lies between tile rows g-1 and g (Fy of NS:393-398)
    for (int k = tid; k < NGY; k += NT) {
        const int col = k % TX, g = k / TX;
        const int L = r_at(col, g - 1), R = r_at(col, g);
        T F[4];   // {mass, v-momentum, u-momentum, energy} from the exchanged call
        ns_hllc(c, s_d[L], s_v[L], s_u[L], s_P[L], s_d[R], s_v[R], s_u[R], s_P[R], F);
        T Gx = F[2], Gy = F[1], GE = F[3];
        if (c.viscous) {   // NS:454-480
            const int gL = g_at(col, g - 1), gR = g_at(col, g);
            const T dudx = T(0.5) * (g_ux[gL] + g_ux[gR]);
            const T dudy = T(0.5) * (g_uy[gL] + g_uy[gR]);
            const T dvdx = T(0.5) * (g_vx[gL] + g_vx[gR]);
            const T dvdy = T(0.5) * (g_vy[gL] + g_vy[gR]);
            const T divv = dudx + dvdy;
            const T tau_yy = c.mu * (T(2.0) * dvdy - (T(2.0) / T(3.0)) * divv);
            const T tau_xy = c.mu * (dudy + dvdx);
            const T uf = T(0.5) * (s_u[L] + s_u[R]);
            const T vf = T(0.5) * (s_v[L] + s_v[R]);
            Gx += -tau_xy;
            Gy += -tau_yy;
            GE += -(uf * tau_xy + vf * tau_yy);
        }
        fy[k] = F[0]; fy[NGY + k] = Gx; fy[2 * NGY + k] = Gy; fy[3 * NGY + k] = GE;
    }
    __syncthreads();

    if (tid >= G::NC) return;
    const int tx = tid % TX, ty = tid / TX;
    const int gi = i0 + tx, gj = j0 + ty;
    if (gi >= c.nx || gj >= c.ny) return;
    const size_t q = (size_t)gj * P + gi;
    // rhs (NS:488-516): flux divergence, then the gravity source with the cell's primitives
    const int kx = ty * (TX + 1) + tx, ky = ty * TX + tx;
    T R[4];
#pragma unroll
    for (int m = 0; m < 4; m++)
        R[m] = -(fx[m * NFX + kx + 1] - fx[m * NFX + kx]) * c.idx1 - (fy[m * NGY + ky + TX] - fy[m * NGY + ky]) * c.idy1;
    if (c.gravity_on) {   // compute_gravity_accel (NS:343-358)
        const int ip = wrap_idx(gi + 1, c.nx), im = wrap_idx(gi - 1, c.nx);
        const int jp = wrap_idx(gj + 1, c.ny), jm = wrap_idx(gj - 1, c.ny);
        const T gx = -(phi[(size_t)gj * P + ip] - phi[(size_t)gj * P + im]) * c.idx2;
        const T gy = -(phi[(size_t)jp * P + gi] - phi[(size_t)jm * P + gi]) * c.idy2;
        const int o = r_at(tx, ty);
        const T d = s_d[o], u = s_u[o], v = s_v[o];
        R[1] += d * gx;
        R[2] += d * gy;
        R[3] += d * (u * gx + v * gy);
    }
    const T dt = (T)(*dtp);
    T nd, nmx, nmy, nE;
    if (!STAGE2) {   // NS:763-771
        nd = in.d[q] + dt * R[0];
        nmx = in.mx[q] + dt * R[1];
        nmy = in.my[q] + dt * R[2];
        nE = in.E[q] + dt * R[3];
        k1.d[q] = R[0]; k1.mx[q] = R[1]; k1.my[q] = R[2]; k1.E[q] = R[3];
    } else {         // NS:774-781
        const T h = T(0.5) * dt;
        nd = un.d[q] + h * (k1.d[q] + R[0]);
        nmx = un.mx[q] + h * (k1.mx[q] + R[1]);
        nmy = un.my[q] + h * (k1.my[q] + R[2]);
        nE = un.E[q] + h * (k1.E[q] + R[3]);
    }
    if (nd < c.floor_rho) nd = c.floor_rho;
    out.d[q] = nd; out.mx[q] = nmx; out.my[q] = nmy; out.E[q] = nE;
}

// compute_dt's reductions (NS:521-533) and the floored-density sum the Poisson
// mean needs (NS:294-296, 372-377): per block max(|u|+a, |v|+a), min rho and
// sum rho of the primitives, FP64 partials.  min/max are order-free; the sum
// has the block_sum tree order.
template <int NT>
__device__ __forceinline__ double ns_block_min(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 1e300;
    if (w == 0) {
        r = (l < NT / 32) ? sh[l] : 1e300;
        for (int o = 16; o > 0; o >>= 1) r = fmin(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;
}

template <class T, int NT>
__global__ void __launch_bounds__(NT)
ns_speed_kernel(const NSConst<T> c, const NSFields<T> s, double* __restrict__ spd_part,
                double* __restrict__ rmin_part, double* __restrict__ rho_part) {
    __shared__ double sh[2 * NT / 32];
    double smax = 0.0, rmin = 1e300, rsum = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const size_t q = (size_t)(k / c.nx) * c.pitch + (k % c.nx);
        const NSPrim<T> W = ns_prim(c, s.d[q], s.mx[q], s.my[q], s.E[q]);
        const T a = ns_sound(c, W);
        const double sx = (double)(fabs(W.u) + a), sy = (double)(fabs(W.v) + a);
        if (sx > smax) smax = sx;   // std::max(smax, x) never keeps a NaN
        if (sy > smax) smax = sy;
        if ((double)W.d < rmin) rmin = (double)W.d;
        rsum += (double)W.d;
    }
    block_max_sum<NT>(smax, rsum, sh);
    const double bmin = ns_block_min<NT>(rmin, sh);
    if (threadIdx.x == 0) { spd_part[blockIdx.x] = smax; rho_part[blockIdx.x] = rsum; rmin_part[blockIdx.x] = bmin; }
}

template <class T, int NT>
__global__ void __launch_bounds__(NT)
ns_rho_sum_kernel(const NSConst<T> c, const T* __restrict__ d, double* __restrict__ rho_part) {
    __shared__ double sh[NT / 32];
    double rsum = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT)
        rsum += (double)vmax(d[(size_t)(k / c.nx) * c.pitch + (k % c.nx)], c.floor_rho);
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) rho_part[blockIdx.x] = bs;
}

// floored copy of the density (the Poisson input W.d, NS:374-377) for a state
// whose density may lie below the floor (an uploaded one: every step floors it)
template <class T>
__global__ void ns_floor_copy_kernel(const NSConst<T> c, const T* __restrict__ d, T* __restrict__ out,
                                     const int* __restrict__ active) {
    if (active && *active == 0) return;
    const size_t n = (size_t)c.nx * c.ny;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const size_t q = (k / c.nx) * c.pitch + (k % c.nx);
        out[q] = vmax(d[q], c.floor_rho);
    }
}

// compute_dt (NS:521-546) from the block partials, then the main loop's
// clamp to t_end (NS:759-760); the loop runs while t < t_end - 1e-14
// (NS:758): past it the step is switched off (active = 0, dt = 0).
struct NSDtSpec {
    double cfl, hmin, mu, cfl_visc, floor_rho, t_end;
    int viscous, clamp_to_end;
};

// D = double (a template: the header is included by several units)
template <class D>
__global__ void ns_dt_kernel(const D* __restrict__ spd_part, const D* __restrict__ rmin_part, int nparts,
                             NSDtSpec d, D* __restrict__ dt_out, const D* __restrict__ t_now,
                             int* __restrict__ active) {
    if (threadIdx.x >= 32 || blockIdx.x != 0) return;
    // one warp: strided shares of the partials, then the lanes combined (max
    // and min are exact, so the order does not matter)
    D smax = 0.0, rho_min = 1e300;
    for (int b = threadIdx.x; b < nparts; b += 32) {
        smax = vmax(smax, spd_part[b]);
        rho_min = vmin(rho_min, rmin_part[b]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        smax = vmax(smax, __shfl_xor_sync(0xffffffffu, smax, o));
        rho_min = vmin(rho_min, __shfl_xor_sync(0xffffffffu, rho_min, o));
    }
    if (threadIdx.x != 0) return;
    const D dt_hyp = (smax > 0.0) ? (d.cfl * d.hmin / smax) : 1e-6;
    D dt = dt_hyp;
    if (d.viscous) {
        const D nu_max = d.mu / vmax(rho_min, (D)d.floor_rho);
        const D dt_visc = (nu_max > 0.0) ? (d.cfl_visc * d.hmin * d.hmin / nu_max) : dt_hyp;
        dt = vmin(dt, dt_visc);
    }
    if (d.clamp_to_end) {
        const D t = *t_now;
        if (!(t < d.t_end - 1e-14)) { active[0] = 0; *dt_out = 0.0; return; }
        if (t + dt > d.t_end) dt = d.t_end - t;
    }
    active[0] = 1;
    *dt_out = dt;
}

// compute_gravity_accel (NS:330-360): g = -(phi[+1] - phi[-1]) / (2 h) as a
// product with the reciprocal, periodic neighbours
template <class T>
__global__ void ns_gravity_kernel(const NSConst<T> c, const T* __restrict__ phi, T* __restrict__ gx,
                                  T* __restrict__ gy) {
    const int n = c.nx * c.ny, P = c.pitch;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = k % c.nx, j = k / c.nx;
        const int ip = wrap_idx(i + 1, c.nx), im = wrap_idx(i - 1, c.nx);
        const int jp = wrap_idx(j + 1, c.ny), jm = wrap_idx(j - 1, c.ny);
        gx[(size_t)j * P + i] = -(phi[(size_t)j * P + ip] - phi[(size_t)j * P + im]) * c.idx2;
        gy[(size_t)j * P + i] = -(phi[(size_t)jp * P + i] - phi[(size_t)jm * P + i]) * c.idy2;
    }
}

// The fields the reference main() stores per snapshot (NS:698-746):
// out[0..7] = rho, P, Mach, u, v, momx, momy, Phi (8 planes of nx*ny doubles)
// from cons_to_prim of each cell; Mach = |v| / a, 0 where a <= 0; Phi from
// the potential of the stored state (0 with gravity off).
template <class T>
__global__ void ns_derived_kernel(const NSConst<T> c, const NSFields<T> s, const T* __restrict__ phi,
                                  double* __restrict__ out) {
    const size_t n = (size_t)c.nx * c.ny;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const size_t q = (k / c.nx) * c.pitch + (k % c.nx);
        const NSPrim<T> W = ns_prim(c, s.d[q], s.mx[q], s.my[q], s.E[q]);
        const T a = ns_sound(c, W);
        const T vmag = sqrt(W.u * W.u + W.v * W.v);
        out[k] = W.d;
        out[n + k] = W.P;
        out[2 * n + k] = (a > T(0.0)) ? (vmag / a) : T(0.0);
        out[3 * n + k] = W.u;
        out[4 * n + k] = W.v;
        out[5 * n + k] = W.d * W.u;
        out[6 * n + k] = W.d * W.v;
        out[7 * n + k] = phi ? (double)phi[q] : 0.0;
    }
}

template <class T, int NT>
__global__ void __launch_bounds__(NT) ns_diag_kernel(const NSConst<T> c, const NSFields<T> s, double* __restrict__ part) {
    __shared__ double sh[NT / 32];
    double acc[4] = {0, 0, 0, 0}, nonf = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const size_t q = (size_t)(k / c.nx) * c.pitch + (k % c.nx);
        const double v[4] = {(double)s.d[q], (double)s.mx[q], (double)s.my[q], (double)s.E[q]};
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
