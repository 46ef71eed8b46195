// Precision-independent kernels of the batched ensemble: per-instance
// reduction finaliser (dt, active flag, density mean) and the device clock.
// Built with -fmad=false, like the single-grid dt finaliser, so that an
// instance's dt rounds exactly like the single-grid path's.
#include "batch_launch.h"

namespace ccb {

// One warp per instance.  Lane l folds the instance's reduce-tile partials
// l, l+32, l+64, ... in order; the 32 lane values are then combined by a
// shuffle-down tree (offsets 16..1).  The density sum therefore has a fixed
// order (restated by the CPU oracle); the CFL maximum is order-free (a NaN
// partial never wins, as in std::max(maxs, x)).  dt as in compute_dt,
// M2:579-598, with the t_end clamp of M2:1114.
__global__ void __launch_bounds__(128)
batch_finalize_kernel(const BatchRed* __restrict__ red, int n, const double* __restrict__ spd_part,
                      const double* __restrict__ rho_part, int flags, double* __restrict__ dt,
                      const double* __restrict__ t, int* __restrict__ active, double* __restrict__ rho_mean) {
    const int id = blockIdx.x * 4 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (id >= n) return;   // whole warps leave together
    const BatchRed r = red[id];
    if (flags & BF_MEAN) {
        double s = 0.0;
        for (int k = lane; k < r.count; k += 32) s = s + rho_part[r.base + k];
        for (int o = 16; o > 0; o >>= 1) s = s + __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) rho_mean[id] = s / r.ncell;
    }
    if (flags & BF_DT) {
        const DtSpec d = r.dts;
        double maxs = d.seed;
        for (int k = lane; k < r.count; k += 32) maxs = vmax(maxs, spd_part[r.base + k]);
        for (int o = 16; o > 0; o >>= 1) maxs = vmax(maxs, __shfl_down_sync(0xffffffffu, maxs, o));
        if (lane != 0) return;
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
    batch_finalize_kernel<<<(n + 3) / 4, 128, 0, s>>>(red, n, spd_part, rho_part, flags, dt, t, active, rho_mean);
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
