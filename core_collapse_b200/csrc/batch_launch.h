// Host-side launchers of the batched-ensemble kernels.  BatchLaunch<T> is
// defined once per precision (batch_f64.cu with -fmad=false, batch_f32.cu with
// the bulk-path flags); DPoissonLaunch<T> in dpoisson.cu (-fmad=false, FP64
// arithmetic with explicit fma); the finaliser and clock in batch_common.cu.
#pragma once
#include <cuda_runtime.h>

#include "batch_kernels.cuh"

namespace ccb {

// A stage tile shape the autotuner may pick.
struct TileShape {
    int tx, ty;
};

template <class T> struct BatchLaunch {
    static int n_shapes();
    static TileShape shape(int k);
    // raise the dynamic shared-memory limit of every candidate (before any launch or capture)
    static cudaError_t prepare();
    // CTAs of candidate k resident per SM
    static cudaError_t resident(int k, int* per_sm);
    static cudaError_t stage(int k, int grid, const BatchInst<T>* inst, const int2* work, int nwork, int src, int dst,
                             bool defer, bool grav, const double* dt, const int* active, cudaStream_t s);
    // stage with the record of the pre-floor update (inst->rec), tile candidate 0, one CTA per tile
    static cudaError_t stage_rec(const BatchInst<T>* inst, const int2* work, int nwork, int src, int dst, bool defer,
                                 bool grav, const double* dt, const int* active, cudaStream_t s);
    static cudaError_t average(const BatchInst<T>* inst, const int2* rwork, int nrwork, int a, int d, int b,
                               const double* dt, const int* active, double* spd_part, double* rho_part,
                               cudaStream_t s);
    static cudaError_t speeds(const BatchInst<T>* inst, const int2* rwork, int nrwork, int src, double* spd_part,
                              double* rho_part, cudaStream_t s);
    static cudaError_t rho_sum(const BatchInst<T>* inst, const int2* rwork, int nrwork, int src, const int* active,
                               double* rho_part, cudaStream_t s);
};

template <class T> struct DPoissonLaunch {
    // shared-memory limit of the tensor-core transforms (FP32; before any launch or capture)
    static cudaError_t prepare();
    // rho of buffer src -> phi, for every active instance
    // gwork: CUDA-core GEMM tiles of gtile x gtile outputs (64 or 32);
    // tcwork: 128 x 128 tiles of the instances solved on the tcgen05 tensor
    // cores (FP32 instances with nx a multiple of 4; a timed-out wait inside
    // them sets *err).  An instance is in one of the two lists.
    static cudaError_t solve(const BatchInst<T>* inst, const int2* gwork, int ngwork, int gtile, const int2* tcwork,
                             int ntcwork, const int2* ywork, int nywork, int src, const double* rho_mean,
                             const int* active, int* err, cudaStream_t s);
};

// flags of the finaliser
constexpr int BF_DT = 1;      // dt and active from the CFL partials
constexpr int BF_MEAN = 2;    // density mean from the density partials
constexpr int BF_CLAMP = 4;   // clamp dt to t_end and set active from t < t_end

cudaError_t launch_batch_finalize(const BatchRed* red, int n, const double* spd_part, const double* rho_part,
                                  int flags, double* dt, const double* t, int* active, double* rho_mean,
                                  cudaStream_t s);
cudaError_t launch_batch_clock(int n, double* t, const double* dt, const int* active, long long* steps,
                               cudaStream_t s);
cudaError_t launch_batch_set_active(int n, int* active, int v, cudaStream_t s);

}  // namespace ccb
