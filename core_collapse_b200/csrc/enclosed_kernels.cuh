// Enclosed-mass radial gravity (compute_enclosed_mass_gravity,
// euler2d_gravity_hllc.cpp:226-286) on the GPU.  The reference sorts the
// cells by distance from the domain centre every call, groups radii within
// 1e-12 of a group's first radius, accumulates the mass in sorted order and
// gives every cell of a group g = -G M_enc / (r^2 + softening^2) along r-hat,
// M_enc = the mass up to the end of its group.  The radii depend only on the
// grid, so the sorted order and each cell's group end are built once on the
// host (cc_euler2d_create); per solve the GPU
//   1. gathers the floored masses in radius order and scans them within
//      blocks of ENC_NT (warp shuffle scans, fixed order)   -- enc_scan_kernel
//   2. scans the block totals (one CTA)                      -- enc_blocks_kernel
//   3. reads M_enc at each group end and writes g            -- enc_gravity_kernel
// FP64 sums throughout; the association of the scan differs from the
// reference's running sum (relative differences at the 1e-16 level).
// The shell-binned provider of gravity_enclosed.h reuses steps 1-2 with the
// cells ordered by shell (enc_shell_gravity_kernel below).
#pragma once
#include "cc_device.cuh"

namespace ccb {

constexpr int ENC_NT = 1024;

// inclusive scan of v over the CTA (ENC_NT threads); sh >= ENC_NT / 32 doubles
__device__ __forceinline__ double enc_block_scan(double v, double* sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += u;
    }
    if (lane == 31) sh[w] = v;
    __syncthreads();
    if (w == 0) {
        double t = (lane < ENC_NT / 32) ? sh[lane] : 0.0;
        for (int o = 1; o < 32; o <<= 1) {
            const double u = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += u;
        }
        sh[lane] = t;   // inclusive totals of warps 0..lane
    }
    __syncthreads();
    if (w > 0) v += sh[w - 1];
    __syncthreads();
    return v;
}

template <class T>
__global__ void __launch_bounds__(ENC_NT)
enc_scan_kernel(const T* __restrict__ rho, int pitch, int nx, const int* __restrict__ order, int n, double floor_rho,
                double cell_area, double* __restrict__ cum, double* __restrict__ blk, const int* __restrict__ active) {
    if (active && *active == 0) return;
    __shared__ double sh[ENC_NT / 32];
    const int t = blockIdx.x * ENC_NT + threadIdx.x;
    double m = 0.0;
    if (t < n) {
        const int k = order[t];
        m = fmax((double)rho[(size_t)(k / nx) * pitch + (k % nx)], floor_rho) * cell_area;
    }
    const double s = enc_block_scan(m, sh);
    if (t < n) cum[t] = s;
    if (threadIdx.x == ENC_NT - 1) blk[blockIdx.x] = s;
}

// exclusive prefix of the nb block totals, in place (one CTA of ENC_NT threads):
// each thread sums a contiguous run in order, the runs are scanned, each
// thread writes its run's prefixes.  D = double (a template: the header is
// included by several units)
template <class D>
__global__ void __launch_bounds__(ENC_NT)
enc_blocks_kernel(D* __restrict__ blk, int nb, const int* __restrict__ active) {
    if (active && *active == 0) return;
    __shared__ double sh[ENC_NT / 32];
    const int per = (nb + ENC_NT - 1) / ENC_NT;
    const int b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
    double s = 0.0;
    for (int b = b0; b < b1; b++) s += blk[b];
    double run = enc_block_scan(s, sh) - s;   // exclusive prefix of this thread's run
    for (int b = b0; b < b1; b++) {
        const double v = blk[b];
        blk[b] = run;
        run += v;
    }
}

template <class T>
__global__ void enc_gravity_kernel(const int* __restrict__ order, const int* __restrict__ gend,
                                   const double* __restrict__ cum, const double* __restrict__ blk, int n, int nx,
                                   int pitch, double x0, double y0, double dx, double dy, double cx, double cy,
                                   double G, double soft2, T* __restrict__ gx, T* __restrict__ gy,
                                   const int* __restrict__ active) {
    if (active && *active == 0) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int e = gend[t] - 1;   // last cell of t's radius group
        const double menc = cum[e] + blk[e / ENC_NT];
        const int k = order[t], i = k % nx, j = k / nx;
        const double rx = (x0 + (i + 0.5) * dx) - cx, ry = (y0 + (j + 0.5) * dy) - cy;
        const double r2 = rx * rx + ry * ry + soft2;
        const double r = sqrt(r2);
        double vx = 0.0, vy = 0.0;
        if (r > 0.0) {
            const double gmag = -G * menc / r2;
            vx = gmag * (rx / r);
            vy = gmag * (ry / r);
        }
        const size_t q = (size_t)j * pitch + i;
        gx[q] = (T)vx;
        gy[q] = (T)vy;
    }
}

// Shell-binned variant (gravity_accel_from_enclosed_mass, gravity_enclosed.h:18-96):
// cells ordered by shell, gend[t] the end of t's shell, so M(<shell) is the
// scan at the shell's end; geo (3 n doubles, sorted order) holds each cell's
// rx, ry and (r^2 + softening^2)^(3/2) from the host.
// g = -G M(<shell) / denom * (rx, ry); 0 where denom <= 0.
template <class T>
__global__ void enc_shell_gravity_kernel(const int* __restrict__ order, const int* __restrict__ gend,
                                         const double* __restrict__ cum, const double* __restrict__ blk,
                                         const double* __restrict__ geo, int n, int nx, int pitch, double G,
                                         T* __restrict__ gx, T* __restrict__ gy, const int* __restrict__ active) {
    if (active && *active == 0) return;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int e = gend[t] - 1;
        const double menc = cum[e] + blk[e / ENC_NT];
        const int k = order[t];
        const double denom = geo[2 * (size_t)n + t];
        double vx = 0.0, vy = 0.0;
        if (!(denom <= 0.0)) {
            const double gcoef = -G * menc / denom;
            vx = gcoef * geo[t];
            vy = gcoef * geo[(size_t)n + t];
        }
        const size_t q = (size_t)(k / nx) * pitch + (k % nx);
        gx[q] = (T)vx;
        gy[q] = (T)vy;
    }
}

}  // namespace ccb
