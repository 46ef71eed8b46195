// Direct Poisson solve for the batched ensemble, in the state precision T
// (FP64 instances: FP64 throughout, bitwise reproducible on the CPU; FP32
// instances: the same operations in FP32).
//
// It solves the discrete problem the reference's SOR iterates towards
// (mhd2d_resistive_hlld_ct_gravity.cpp:207-223: 5-point Laplacian, clamp or
// wrap neighbours, zero-mean potential) exactly instead of iterating:
//   1. U = R * Tx^T     R = 4 pi G (rho - mean), Tx rows = orthonormal
//                       eigenvectors of the x second difference (DCT-II for
//                       clamp, Hartley for periodic)        -- dp_gemm, MODE 0
//   2. per x wavenumber k: (Dyy + lam_x[k]) u_k = U[:, k] along y: Thomas,
//      cyclic Thomas (Sherman-Morrison), or for k = 0 the cumulative-flux
//      solution with its mean removed                        -- dp_ysolve
//   3. phi = U * Tx                                          -- dp_gemm, MODE 1
// The translation unit is compiled with -fmad=false and every multiply-add is
// an explicit fma() in a fixed order, so the CPU restatement (std::fma in the
// same order) reproduces the result bit for bit.
//
// Work-lists: GEMM tiles {instance, (tm << 16) | tn} of TM x TM outputs (TM 64,
// or 32 when 64-tiles would leave SMs idle: same per-output k order, same bits);
// y-solve items {instance, -1} (the singular wavenumber 0) and {instance,
// column block} of DPC wavenumbers 1 + DPC cb + lane, one thread per column.
#pragma once
#include <type_traits>

#include "batch_kernels.cuh"

namespace ccb {

constexpr int DPK = 16, DPNT = 256;   // GEMM K chunk and threads; tiles TM x TM, TM/16 x TM/16 outputs per thread
constexpr int DPC = 32;                                    // y-solve columns per block

// Software-pipelined tile loop: the next K chunk is loaded into registers
// while the current one is multiplied from shared memory; raw values are
// converted (MODE 0: 4 pi G (rho - mean)) only when they are stored, so no
// instruction waits on a load in flight during the multiply.
template <class T, int MODE, int TM>
__global__ void __launch_bounds__(DPNT)
dp_gemm_kernel(const BatchInst<T>* __restrict__ inst, const int2* __restrict__ gwork, int ngwork, int src,
               const double* __restrict__ rho_mean, const int* __restrict__ active) {
    constexpr int RPT = TM / 16;            // outputs per thread per dimension
    constexpr int LQ = TM * DPK / DPNT;     // tile elements each thread loads per K chunk
    __shared__ T As[DPK][TM + 1];           // k-major A tile
    __shared__ T Bs[DPK][TM];
    const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
    for (int w = blockIdx.x; w < ngwork; w += gridDim.x) {
        const int2 it = gwork[w];
        if (active[it.x] == 0) continue;   // uniform over the block
        const BatchInst<T>& I = inst[it.x];
        const int nx = I.c.nx, ny = I.c.ny, P = I.c.pitch;
        const int m0 = (it.y >> 16) * TM, n0 = (it.y & 0xffff) * TM;
        const T* __restrict__ B = (MODE == 0) ? I.txt : I.tx;   // K x N row-major, K = N = nx
        const T* __restrict__ rho = I.buf[src].rho;
        const T* __restrict__ ah = I.ah;
        const T mean = (MODE == 0) ? (T)rho_mean[it.x] : T(0);
        const T fpg = (T)I.fourpiG;
        T ra[LQ];
        T rb[LQ];
        auto gload = [&](int k0) {
#pragma unroll
            for (int q = 0; q < LQ; q++) {
                const int e = threadIdx.x + q * DPNT;
                const int gm = m0 + e / DPK, gk = k0 + e % DPK;
                ra[q] = T(0);
                if (gm < ny && gk < nx) {
                    if (MODE == 0) ra[q] = rho[(size_t)gm * P + gk];
                    else ra[q] = ah[(size_t)gm * nx + gk];
                }
                const int gkb = k0 + e / TM, gn = n0 + e % TM;
                rb[q] = (gkb < nx && gn < nx) ? B[(size_t)gkb * nx + gn] : T(0);
            }
        };
        T acc[RPT][RPT];
#pragma unroll
        for (int r = 0; r < RPT; r++)
#pragma unroll
            for (int c = 0; c < RPT; c++) acc[r][c] = T(0);
        gload(0);
        for (int k0 = 0; k0 < nx; k0 += DPK) {
#pragma unroll
            for (int q = 0; q < LQ; q++) {
                const int e = threadIdx.x + q * DPNT;
                const int m = e / DPK, kk = e % DPK;
                T v = ra[q];
                if (MODE == 0) v = (m0 + m < ny && k0 + kk < nx) ? fpg * (v - mean) : T(0);
                As[kk][m] = v;
                Bs[e / TM][e % TM] = rb[q];
            }
            __syncthreads();
            if (k0 + DPK < nx) gload(k0 + DPK);
            const int kend = min(DPK, nx - k0);
            for (int kk = 0; kk < kend; kk++) {
                T a[RPT], b[RPT];
#pragma unroll
                for (int r = 0; r < RPT; r++) a[r] = As[kk][tr + 16 * r];
#pragma unroll
                for (int c = 0; c < RPT; c++) b[c] = Bs[kk][tc + 16 * c];
#pragma unroll
                for (int r = 0; r < RPT; r++)
#pragma unroll
                    for (int c = 0; c < RPT; c++) acc[r][c] = fma(a[r], b[c], acc[r][c]);
            }
            __syncthreads();
        }
#pragma unroll
        for (int r = 0; r < RPT; r++) {
            const int gm = m0 + tr + 16 * r;
            if (gm >= ny) continue;
#pragma unroll
            for (int c = 0; c < RPT; c++) {
                const int gn = n0 + tc + 16 * c;
                if (gn >= nx) continue;
                if (MODE == 0) I.ah[(size_t)gm * nx + gn] = acc[r][c];
                else I.phi[(size_t)gm * P + gn] = acc[r][c];
            }
        }
    }
}

// y solves: one thread per x wavenumber k >= 1 (a warp covers 32 adjacent
// wavenumbers, so every row access is one coalesced 256-byte line), the
// singular k = 0 on a CTA of its own.  Each sweep is a chain of fma's whose
// loads do not depend on the chain: rows are fetched YB at a time into
// registers one block ahead of the block being computed, which overlaps the
// L2 latency with the chain.  The arithmetic and its order are those of the
// CPU restatement (bitwise).
constexpr int YB = 16;

// forward sweep: d_0 = u_0 inv_0, d_j = (u_j - a d_{j-1}) inv_j, u_j <- d_j; returns d_{n-1}
// (the prefetch of the block after the last one reads clamped, in-range rows)
template <class S_>
__device__ __forceinline__ S_ ysweep_fwd(S_* __restrict__ u, const S_* __restrict__ inv, size_t S, int n, S_ a) {
    S_ d = u[0] * inv[0];
    u[0] = d;
    int j = 1;
    const int nb = (n - 1) / YB;
    S_ cu[YB], ci[YB];
#pragma unroll
    for (int t = 0; t < YB; t++) {
        const int r = min(j + t, n - 1);
        cu[t] = u[r * S]; ci[t] = inv[r * S];
    }
    for (int b = 0; b < nb; b++, j += YB) {
        S_ nu[YB], ni[YB];
#pragma unroll
        for (int t = 0; t < YB; t++) {
            const int r = min(j + YB + t, n - 1);
            nu[t] = u[r * S]; ni[t] = inv[r * S];
        }
#pragma unroll
        for (int t = 0; t < YB; t++) {
            d = fma(-a, d, cu[t]) * ci[t];
            u[(j + t) * S] = d;
        }
#pragma unroll
        for (int t = 0; t < YB; t++) { cu[t] = nu[t]; ci[t] = ni[t]; }
    }
    for (; j < n; j++) {
        d = fma(-a, d, u[j * S]) * inv[j * S];
        u[j * S] = d;
    }
    return d;
}

// backward sweep: x_{n-1} = d_{n-1}, x_j = d_j - cp_j x_{j+1}, u_j <- x_j; returns x_0
template <class S_>
__device__ __forceinline__ S_ ysweep_bwd(S_* __restrict__ u, const S_* __restrict__ cp, size_t S, int n, S_ x) {
    int j = n - 2;
    const int nb = (n - 1) / YB;
    S_ cu[YB], cc[YB];
#pragma unroll
    for (int t = 0; t < YB; t++) {
        const int r = max(j - t, 0);
        cu[t] = u[r * S]; cc[t] = cp[r * S];
    }
    for (int b = 0; b < nb; b++, j -= YB) {
        S_ nu[YB], nc[YB];
#pragma unroll
        for (int t = 0; t < YB; t++) {
            const int r = max(j - YB - t, 0);
            nu[t] = u[r * S]; nc[t] = cp[r * S];
        }
#pragma unroll
        for (int t = 0; t < YB; t++) {
            x = fma(-cc[t], x, cu[t]);
            u[(j - t) * S] = x;
        }
#pragma unroll
        for (int t = 0; t < YB; t++) { cu[t] = nu[t]; cc[t] = nc[t]; }
    }
    for (; j >= 0; j--) {
        x = fma(-cp[j * S], x, u[j * S]);
        u[j * S] = x;
    }
    return x;
}

template <class T>
__global__ void __launch_bounds__(DPC)
dp_ysolve_kernel(const BatchInst<T>* __restrict__ inst, const int2* __restrict__ ywork, int nywork,
                 const int* __restrict__ active) {
    for (int w = blockIdx.x; w < nywork; w += gridDim.x) {
        const int2 it = ywork[w];
        if (active[it.x] == 0) continue;
        const BatchInst<T>& I = inst[it.x];
        const int nx = I.c.nx, n = I.c.ny;
        const size_t S = (size_t)nx;
        const bool py = I.c.ay.periodic != 0;
        const T a = (T)I.ay;
        if (it.y < 0) {
            // singular k = 0: flux G_j = a (u_{j+1} - u_j) = G_{j-1} + r_j, then mean removal
            if (threadIdx.x != 0) continue;
            T* __restrict__ u = I.ah;
            T g0 = T(0);
            if (py) {
                T Sr = T(0), SS = T(0);
#pragma unroll 16
                for (int j = 0; j < n; j++) { Sr = Sr + u[j * S]; SS = SS + Sr; }
                g0 = -(SS / (T)n);
            }
            const T dy2 = (T)I.dy2;
            T G = g0, prev = T(0);
            T r = u[0];
            u[0] = T(0);
#pragma unroll 16
            for (int j = 0; j + 1 < n; j++) {
                G = G + r;
                r = u[(j + 1) * S];
                prev = fma(dy2, G, prev);
                u[(j + 1) * S] = prev;
            }
            T m = T(0);
#pragma unroll 16
            for (int j = 0; j < n; j++) m = m + u[j * S];
            m = m / (T)n;
#pragma unroll 16
            for (int j = 0; j < n; j++) u[j * S] = u[j * S] - m;
            continue;
        }
        const int col = 1 + it.y * DPC + threadIdx.x;
        if (col >= nx) continue;
        T* __restrict__ u = I.ah + col;
        const T d = ysweep_fwd<T>(u, I.yinv + col, S, n, a);
        const T x = ysweep_bwd<T>(u, I.ycp + col, S, n, d);
        if (!py) continue;
        const T* __restrict__ z = I.yz + col;
        const T gam = -fma(T(-2), a, I.lamx[col]);
        const T fac = fma(a / gam, d, x) * I.yfden[col];   // d = x_{n-1}, x = x_0
#pragma unroll 8
        for (int j = 0; j < n; j++) u[j * S] = fma(-fac, z[j * S], u[j * S]);
    }
}

}  // namespace ccb
