// Definitions of NSLaunch<T>; included once per precision TU.
#pragma once
#include "ns2d_launch.h"

namespace ccb {

template <class T>
cudaError_t NSLaunch<T>::prepare() {
    const int smem = (int)NSGeom<T>::smem;
    cudaError_t e = cudaFuncSetAttribute(ns_stage_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(ns_stage_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <class T>
cudaError_t NSLaunch<T>::stage(const NSConst<T>& c, const NSFields<T>& un, const NSFields<T>& in,
                               const NSFields<T>& k1, const NSFields<T>& out, bool stage2, const T* phi,
                               const double* dt, const int* active, cudaStream_t s) {
    using G = NSGeom<T>;
    dim3 grid((c.nx + G::TX - 1) / G::TX, (c.ny + G::TY - 1) / G::TY);
    if (stage2) ns_stage_kernel<T, true><<<grid, G::NT, G::smem, s>>>(c, un, in, k1, out, phi, dt, active);
    else ns_stage_kernel<T, false><<<grid, G::NT, G::smem, s>>>(c, un, in, k1, out, phi, dt, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t NSLaunch<T>::speeds(const NSConst<T>& c, const NSFields<T>& st, double* spd_part, double* rmin_part,
                                double* rho_part, cudaStream_t s) {
    ns_speed_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, st, spd_part, rmin_part, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t NSLaunch<T>::rho_sum(const NSConst<T>& c, const T* d, double* rho_part, cudaStream_t s) {
    ns_rho_sum_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, d, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t NSLaunch<T>::floor_copy(const NSConst<T>& c, const T* d, T* out, const int* active, cudaStream_t s) {
    size_t g = ((size_t)c.nx * c.ny + 255) / 256;
    if (g > 4096) g = 4096;
    ns_floor_copy_kernel<T><<<(int)g, 256, 0, s>>>(c, d, out, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t NSLaunch<T>::gravity(const NSConst<T>& c, const T* phi, T* gx, T* gy, cudaStream_t s) {
    int g = (c.nx * c.ny + 255) / 256;
    if (g > 4096) g = 4096;
    ns_gravity_kernel<T><<<g, 256, 0, s>>>(c, phi, gx, gy);
    return cudaGetLastError();
}

template <class T>
cudaError_t NSLaunch<T>::diag(const NSConst<T>& c, const NSFields<T>& st, double* part, cudaStream_t s) {
    ns_diag_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, st, part);
    return cudaGetLastError();
}

template <class T>
cudaError_t NSLaunch<T>::derived(const NSConst<T>& c, const NSFields<T>& st, const T* phi, double* out,
                                 cudaStream_t s) {
    size_t g = ((size_t)c.nx * c.ny + 255) / 256;
    if (g > 4096) g = 4096;
    ns_derived_kernel<T><<<(int)g, 256, 0, s>>>(c, st, phi, out);
    return cudaGetLastError();
}

}  // namespace ccb
