// FP64 instantiation of the 2D Navier-Stokes kernels (the parity path;
// -fmad=false), and the dt kernel's launcher.
#include "ns2d_impl.cuh"

namespace ccb {
template struct NSLaunch<double>;

cudaError_t launch_ns_dt(const double* spd_part, const double* rmin_part, NSDtSpec d, double* dt_out,
                         const double* t_now, int* active, cudaStream_t s) {
    ns_dt_kernel<double><<<1, 32, 0, s>>>(spd_part, rmin_part, RED_BLOCKS, d, dt_out, t_now, active);
    return cudaGetLastError();
}
}  // namespace ccb
