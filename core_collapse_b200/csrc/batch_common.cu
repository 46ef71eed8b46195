// Precision-independent kernels of the batched ensemble: per-instance
// reduction finaliser (dt, active flag, density mean) and the device clock.
// Built with -fmad=false, like the single-grid dt finaliser, so that an
// instance's dt rounds exactly like the single-grid path's.
#include "batch_launch.h"

namespace ccb {

// One thread per instance.  The CFL maximum and the density sum run over the
// instance's reduce-tile partials in tile order (compute_dt, M2:579-598, with
// the t_end clamp of M2:1114).
__global__ void batch_finalize_kernel(const BatchRed* __restrict__ red, int n, const double* __restrict__ spd_part,
                                      const double* __restrict__ rho_part, int flags, double* __restrict__ dt,
                                      const double* __restrict__ t, int* __restrict__ active,
                                      double* __restrict__ rho_mean) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= n) return;
    const BatchRed r = red[id];
    if (flags & BF_MEAN) {
        double s = 0.0;
#pragma unroll 16
        for (int k = 0; k < r.count; k++) s += rho_part[r.base + k];
        rho_mean[id] = s / r.ncell;
    }
    if (flags & BF_DT) {
        const DtSpec d = r.dts;
        double maxs = d.seed;
#pragma unroll 16
        for (int k = 0; k < r.count; k++) maxs = vmax(maxs, spd_part[r.base + k]);
        const double dt_h = d.cfl * d.hmin / maxs;
        double v = dt_h;
        if (d.cap) {
            double dt_r = 1e100;
            if (d.eta > 0.0) dt_r = 0.25 * d.hmin * d.hmin / d.eta;
            v = vmin(dt_h, dt_r);
        }
        if (flags & BF_CLAMP) {
            const double tt = t[id];
            if (!(tt < d.t_end - d.end_eps)) { active[id] = 0; dt[id] = 0.0; return; }
            if (tt + v > d.t_end) v = d.t_end - tt;
        }
        active[id] = 1;
        dt[id] = v;
    }
}

__global__ void batch_clock_kernel(int n, double* __restrict__ t, const double* __restrict__ dt,
                                   const int* __restrict__ active, long long* __restrict__ steps) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < n && active[id]) { t[id] = t[id] + dt[id]; steps[id] = steps[id] + 1; }
}

__global__ void batch_set_active_kernel(int n, int* __restrict__ active, int v) {
    const int id = blockIdx.x * blockDim.x + threadIdx.x;
    if (id < n) active[id] = v;
}

cudaError_t launch_batch_finalize(const BatchRed* red, int n, const double* spd_part, const double* rho_part,
                                  int flags, double* dt, const double* t, int* active, double* rho_mean,
                                  cudaStream_t s) {
    batch_finalize_kernel<<<(n + 127) / 128, 128, 0, s>>>(red, n, spd_part, rho_part, flags, dt, t, active, rho_mean);
    return cudaGetLastError();
}

cudaError_t launch_batch_clock(int n, double* t, const double* dt, const int* active, long long* steps,
                               cudaStream_t s) {
    batch_clock_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, t, dt, active, steps);
    return cudaGetLastError();
}

cudaError_t launch_batch_set_active(int n, int* active, int v, cudaStream_t s) {
    batch_set_active_kernel<<<(n + 127) / 128, 128, 0, s>>>(n, active, v);
    return cudaGetLastError();
}

}  // namespace ccb
