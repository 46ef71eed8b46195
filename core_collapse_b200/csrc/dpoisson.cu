// Launchers of the batched direct Poisson solve, both state precisions.
// Built with -fmad=false: every multiply-add is an explicit fma().
#include "batch_launch.h"
#include "dpoisson_kernels.cuh"

namespace ccb {

template <class T>
cudaError_t DPoissonLaunch<T>::solve(const BatchInst<T>* inst, const int2* gwork, int ngwork, int gtile,
                                     const int2* ywork, int nywork, int src, const double* rho_mean,
                                     const int* active, cudaStream_t s) {
    cudaError_t e;
    if (gtile == 32) dp_gemm_kernel<T, 0, 32><<<ngwork, DPNT, 0, s>>>(inst, gwork, ngwork, src, rho_mean, active);
    else dp_gemm_kernel<T, 0, 64><<<ngwork, DPNT, 0, s>>>(inst, gwork, ngwork, src, rho_mean, active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    dp_ysolve_kernel<T><<<nywork, DPC, 0, s>>>(inst, ywork, nywork, active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (gtile == 32) dp_gemm_kernel<T, 1, 32><<<ngwork, DPNT, 0, s>>>(inst, gwork, ngwork, src, rho_mean, active);
    else dp_gemm_kernel<T, 1, 64><<<ngwork, DPNT, 0, s>>>(inst, gwork, ngwork, src, rho_mean, active);
    return cudaGetLastError();
}

template struct DPoissonLaunch<double>;
template struct DPoissonLaunch<float>;

}  // namespace ccb
