// Host-side launchers of the 3D MHD kernels, defined once per precision in
// mhd3d_f64.cu (-fmad=false, the parity path) and mhd3d_f32.cu.
#pragma once
#include <cuda_runtime.h>

#include "mhd2d_launch.h"
#include "mhd3d_kernels.cuh"

namespace ccb {

template <class T> struct M3Launch {
    // defer: the deferred Joule step first (its cell-centred B of s into bcc, then the pass)
    static cudaError_t prim(const M3Const<T>& c, const Fields3<T>& s, const PrimData<T>& pr, bool defer,
                            const Bcc3<T>& bcc, const double* dt, const int* active, cudaStream_t st);
    static cudaError_t faces(const M3Const<T>& c, const Fields3<T>& s, const PrimData<T>& pr, const FaceData<T>& X,
                             const FaceData<T>& Y, const FaceData<T>& Z, const int* active, cudaStream_t st);
    static cudaError_t update(const M3Const<T>& c, const Fields3<T>& in, const Fields3<T>& out, const FaceData<T>& X,
                              const FaceData<T>& Y, const FaceData<T>& Z, const double* dt, const int* active,
                              cudaStream_t st);
    // edge EMFs and the CT face update in one pass (m3_emf_ct_kernel)
    static cudaError_t emf_ct(const M3Const<T>& c, const Fields3<T>& in, const Fields3<T>& out, const FaceData<T>& X,
                              const FaceData<T>& Y, const FaceData<T>& Z, const double* dt, const int* active,
                              cudaStream_t st);
    // bcc: scratch planes for the cell-centred B of s2 (its Joule step)
    static cudaError_t average(const M3Const<T>& c, const Fields3<T>& un, const Fields3<T>& s2, const Fields3<T>& out,
                               const Bcc3<T>& bcc, const double* dt, const int* active, double* spd_part,
                               double* rho_part, cudaStream_t st);
    static cudaError_t speeds(const M3Const<T>& c, const Fields3<T>& s, double* spd_part, cudaStream_t st);
    static cudaError_t diag(const M3Const<T>& c, const Fields3<T>& s, double* part, cudaStream_t st);
    // the 11 snapshot fields of the reference's store, out: 11 planes of nx*ny*nz doubles
    static cudaError_t derived(const M3Const<T>& c, const Fields3<T>& s, double* out, cudaStream_t st);
    static cudaError_t pack_in(const double* src, T* dst, int w, int h, int d, int P, long long PS, cudaStream_t st);
    static cudaError_t pack_out(const T* src, double* dst, int w, int h, int d, int P, long long PS, cudaStream_t st);
};

}  // namespace ccb
