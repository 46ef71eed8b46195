// Definitions of M3Launch<T>; included once per precision TU.
#pragma once
#include "mhd3d_launch.h"

namespace ccb {

namespace {
inline int grid3(long long n) {
    long long g = (n + 255) / 256;
    if (g < 1) g = 1;
    if (g > 148LL * 16) g = 148LL * 16;
    return (int)g;
}
}  // namespace

template <class T>
cudaError_t M3Launch<T>::prim(const M3Const<T>& c, const Fields3<T>& s, const PrimData<T>& pr, bool defer,
                              const Bcc3<T>& bcc, const double* dt, const int* active, cudaStream_t st) {
    const int g = grid3((long long)c.nx * c.ny * c.nz);
    if (defer && c.resistive) {
        m3_bcc_kernel<T><<<g, 256, 0, st>>>(c, s, bcc, active);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (defer) m3_prim_kernel<T, true><<<g, 256, 0, st>>>(c, s, pr, bcc, dt, active);
    else m3_prim_kernel<T, false><<<g, 256, 0, st>>>(c, s, pr, bcc, dt, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::faces(const M3Const<T>& c, const Fields3<T>& s, const PrimData<T>& pr, const FaceData<T>& X,
                               const FaceData<T>& Y, const FaceData<T>& Z, const int* active, cudaStream_t st) {
    m3_face_kernel<T, 0><<<grid3((long long)(c.nx + 1) * c.ny * c.nz), 256, 0, st>>>(c, s, pr, X, active);
    if constexpr (sizeof(T) == 4) {   // FP32: y and z faces as marches (FP64's window needs ~170 registers)
        const dim3 gy((c.nx + 31) / 32, (c.nz + 7) / 8, (c.ny + 1 + M3_FACE_MCH - 1) / M3_FACE_MCH);
        m3_face_march_kernel<T, 1><<<gy, 256, 0, st>>>(c, s, pr, Y, active);
        const dim3 gz((c.nx + 31) / 32, (c.ny + 7) / 8, (c.nz + 1 + M3_FACE_MCH - 1) / M3_FACE_MCH);
        m3_face_march_kernel<T, 2><<<gz, 256, 0, st>>>(c, s, pr, Z, active);
    } else {
        m3_face_kernel<T, 1><<<grid3((long long)c.nx * (c.ny + 1) * c.nz), 256, 0, st>>>(c, s, pr, Y, active);
        m3_face_kernel<T, 2><<<grid3((long long)c.nx * c.ny * (c.nz + 1)), 256, 0, st>>>(c, s, pr, Z, active);
    }
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::update(const M3Const<T>& c, const Fields3<T>& in, const Fields3<T>& out, const FaceData<T>& X,
                                const FaceData<T>& Y, const FaceData<T>& Z, const double* dt, const int* active,
                                cudaStream_t st) {
    m3_update_kernel<T><<<grid3((long long)c.nx * c.ny * c.nz), 256, 0, st>>>(c, in, out, X, Y, Z, dt, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::emf_ct(const M3Const<T>& c, const Fields3<T>& in, const Fields3<T>& out, const FaceData<T>& X,
                                const FaceData<T>& Y, const FaceData<T>& Z, const double* dt, const int* active,
                                cudaStream_t st) {
    const dim3 g((c.nx + 1 + 30) / 31, (c.ny + 1 + 6) / 7, (c.nz + 1 + M3_EDGE_KCH - 1) / M3_EDGE_KCH);
    m3_emf_ct_kernel<T><<<g, 256, 0, st>>>(c, in, out, X, Y, Z, dt, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::average(const M3Const<T>& c, const Fields3<T>& un, const Fields3<T>& s2, const Fields3<T>& out,
                                 const Bcc3<T>& bcc, const double* dt, const int* active, double* spd_part,
                                 double* rho_part, cudaStream_t st) {
    if (c.resistive) {
        m3_bcc_kernel<T><<<grid3((long long)c.nx * c.ny * c.nz), 256, 0, st>>>(c, s2, bcc, active);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    m3_average_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, st>>>(c, un, s2, out, bcc, dt, active, spd_part, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::speeds(const M3Const<T>& c, const Fields3<T>& s, double* spd_part, cudaStream_t st) {
    m3_speed_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, st>>>(c, s, spd_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::diag(const M3Const<T>& c, const Fields3<T>& s, double* part, cudaStream_t st) {
    m3_diag_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, st>>>(c, s, part);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::derived(const M3Const<T>& c, const Fields3<T>& s, double* out, cudaStream_t st) {
    size_t g = ((size_t)c.nx * c.ny * c.nz + 255) / 256;
    if (g > 8192) g = 8192;
    m3_derived_kernel<T><<<(int)g, 256, 0, st>>>(c, s, out);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::pack_in(const double* src, T* dst, int w, int h, int d, int P, long long PS, cudaStream_t st) {
    pack3_in_kernel<T><<<grid3((long long)w * h * d), 256, 0, st>>>(src, dst, w, h, d, P, PS);
    return cudaGetLastError();
}

template <class T>
cudaError_t M3Launch<T>::pack_out(const T* src, double* dst, int w, int h, int d, int P, long long PS,
                                  cudaStream_t st) {
    pack3_out_kernel<T><<<grid3((long long)w * h * d), 256, 0, st>>>(src, dst, w, h, d, P, PS);
    return cudaGetLastError();
}

}  // namespace ccb
