// Precision-independent kernels and launchers: dt finalisation, the device
// clock, and the cooperative red-black SOR.  Built with -fmad=false (FP64
// arithmetic that must round like the reference).
#include "mhd2d_launch.h"

namespace ccb {

__global__ void m2_dt_finalize_kernel(const double* __restrict__ spd_part, int nparts, DtSpec d,
                                      double* __restrict__ dt_out, const double* __restrict__ t_now,
                                      int* __restrict__ active) {
    if (threadIdx.x >= 32 || blockIdx.x != 0) return;
    // one warp: each lane folds a strided share of the partials into the seed
    // (a NaN partial never wins), then the lanes' maxima are combined; max is
    // exact, so the order does not matter
    double maxs = d.seed;
    for (int b = threadIdx.x; b < nparts; b += 32) maxs = vmax(maxs, spd_part[b]);
    for (int o = 16; o > 0; o >>= 1) maxs = vmax(maxs, __shfl_xor_sync(0xffffffffu, maxs, o));
    if (threadIdx.x != 0) return;
    const double dt_h = d.cfl * d.hmin / maxs;
    double dt = dt_h;
    if (d.cap) {
        double dt_r = 1e100;
        if (d.eta > 0.0) dt_r = 0.25 * d.hmin * d.hmin / d.eta;
        dt = vmin(dt_h, dt_r);
    }
    if (d.clamp_to_end) {
        const double t = *t_now;
        if (!(t < d.t_end - d.end_eps)) { active[0] = 0; *dt_out = 0.0; return; }
        if (d.check && !(isfinite(dt) && dt > 0.0)) { active[0] = 0; active[3] = 1; *dt_out = 0.0; return; }
        if (t + dt > d.t_end) dt = d.t_end - t;
    }
    active[0] = 1;
    *dt_out = dt;
}

__global__ void m2_clock_kernel(double* __restrict__ t, const double* __restrict__ dt, const int* __restrict__ active,
                                long long* __restrict__ steps) {
    if (threadIdx.x == 0 && blockIdx.x == 0 && *active) { *t = *t + *dt; *steps = *steps + 1; }
}

__global__ void set_scalar_kernel(double* p, double v) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *p = v;
}

cudaError_t launch_dt_finalize(const double* spd_part, DtSpec d, double* dt_out, const double* t_now, int* active,
                               cudaStream_t s) {
    m2_dt_finalize_kernel<<<1, 32, 0, s>>>(spd_part, RED_BLOCKS, d, dt_out, t_now, active);
    return cudaGetLastError();
}

cudaError_t launch_clock(double* t, const double* dt, const int* active, long long* steps, cudaStream_t s) {
    m2_clock_kernel<<<1, 32, 0, s>>>(t, dt, active, steps);
    return cudaGetLastError();
}

cudaError_t launch_set_scalar(double* p, double v, cudaStream_t s) {
    set_scalar_kernel<<<1, 32, 0, s>>>(p, v);
    return cudaGetLastError();
}

constexpr int SOR_NT = 1024;

cudaError_t launch_sor(const SorArgs& a, int* nblocks_out, cudaStream_t s) {
    int dev = 0, nsm = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sor_rb_kernel<SOR_NT>, SOR_NT, 0)) != cudaSuccess)
        return e;
    if (per_sm < 1) return cudaErrorLaunchOutOfResources;
    // enough blocks to cover half the grid per colour, at most one wave
    const int ncell = a.nx * a.ny;
    int want = (ncell / 2 + SOR_NT - 1) / SOR_NT;
    if (want < 1) want = 1;
    int cap = nsm;   // one 1024-thread CTA per SM: the sweeps are grid-barrier bound, and fewer, larger CTAs arrive faster
    int nb = want < cap ? want : cap;
    if (nblocks_out) *nblocks_out = nb;
    SorArgs args = a;
    void* params[] = {&args};
    return cudaLaunchCooperativeKernel((const void*)sor_rb_kernel<SOR_NT>, dim3(nb), dim3(SOR_NT), params, 0, s);
}

constexpr int SOR_LEX_NT = 1024;

template <class T>
cudaError_t launch_sor_lex(const SorLexArgs& a, const T* rho, cudaStream_t s) {
    sor_lex_kernel<T, SOR_LEX_NT><<<1, SOR_LEX_NT, 0, s>>>(a, rho);
    return cudaGetLastError();
}
template cudaError_t launch_sor_lex<float>(const SorLexArgs&, const float*, cudaStream_t);
template cudaError_t launch_sor_lex<double>(const SorLexArgs&, const double*, cudaStream_t);

}  // namespace ccb
