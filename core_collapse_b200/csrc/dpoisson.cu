// Launchers of the batched direct Poisson solve, both state precisions.
// Built with -fmad=false: every multiply-add is an explicit fma().
#include <type_traits>

#include "batch_launch.h"
#include "dpoisson_kernels.cuh"
#include "dpoisson_tc.cuh"

namespace ccb {

template <class T> cudaError_t DPoissonLaunch<T>::prepare() {
    if constexpr (sizeof(T) == 4) {
        cudaError_t e = cudaFuncSetAttribute(dp_gemm_tc_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
        if (e != cudaSuccess) return e;
        return cudaFuncSetAttribute(dp_gemm_tc_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    }
    return cudaSuccess;
}

template <class T>
cudaError_t DPoissonLaunch<T>::solve(const BatchInst<T>* inst, const int2* gwork, int ngwork, int gtile,
                                     const int2* tcwork, int ntcwork, const int2* ywork, int nywork, int src,
                                     const double* rho_mean, const int* active, int* err, cudaStream_t s) {
    cudaError_t e;
    if (gtile != 64 && gtile != 32) return cudaErrorInvalidValue;
    if constexpr (sizeof(T) != 4) {
        if (ntcwork > 0) return cudaErrorInvalidValue;
    }
    auto gemm = [&](auto mode) -> cudaError_t {
        constexpr int MODE = decltype(mode)::value;
        if constexpr (sizeof(T) == 4) {
            if (ntcwork > 0) {
                dp_gemm_tc_kernel<MODE><<<ntcwork, TCNT, TC_SMEM, s>>>(inst, tcwork, src, rho_mean, active, err);
                cudaError_t r = cudaGetLastError();
                if (r != cudaSuccess) return r;
            }
        }
        if (ngwork > 0) {
            if (gtile == 32) dp_gemm_kernel<T, MODE, 32><<<ngwork, DPNT, 0, s>>>(inst, gwork, ngwork, src, rho_mean, active);
            else dp_gemm_kernel<T, MODE, 64><<<ngwork, DPNT, 0, s>>>(inst, gwork, ngwork, src, rho_mean, active);
        }
        return cudaGetLastError();
    };
    if ((e = gemm(std::integral_constant<int, 0>())) != cudaSuccess) return e;
    dp_ysolve_kernel<T><<<nywork, DPC, 0, s>>>(inst, ywork, nywork, active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    return gemm(std::integral_constant<int, 1>());
}

template struct DPoissonLaunch<double>;
template struct DPoissonLaunch<float>;

}  // namespace ccb
