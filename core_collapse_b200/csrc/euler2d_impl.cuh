// Definitions of EHLaunch<T>; included once per precision TU.
#pragma once
#include "euler2d_launch.h"

namespace ccb {

template <class T>
cudaError_t EHLaunch<T>::prepare() {
    const int smem = (int)EHGeom<T>::smem;
    cudaError_t e = cudaFuncSetAttribute(eh_stage_kernel<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(eh_stage_kernel<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

template <class T>
cudaError_t EHLaunch<T>::stage(const EHConst<T>& c, const EHFields<T>& un, const EHFields<T>& in,
                               const EHFields<T>& out, bool stage2, const T* phi, const T* gxa, const T* gya,
                               const double* dt, const int* active, cudaStream_t s) {
    using G = EHGeom<T>;
    dim3 grid((c.nx + G::TX - 1) / G::TX, (c.ny + G::TY - 1) / G::TY);
    if (stage2) eh_stage_kernel<T, true><<<grid, G::NT, G::smem, s>>>(c, un, in, out, phi, gxa, gya, dt, active);
    else eh_stage_kernel<T, false><<<grid, G::NT, G::smem, s>>>(c, un, in, out, phi, gxa, gya, dt, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t EHLaunch<T>::enclosed(const EHConst<T>& c, const T* rho, const int* order, const int* gend, int n,
                                  double* cum, double* blk, double x0, double y0, double dx, double dy, double cx,
                                  double cy, double G, double soft2, double floor_rho, T* gx, T* gy,
                                  const int* active, cudaStream_t s) {
    const int nb = (n + ENC_NT - 1) / ENC_NT;
    enc_scan_kernel<T><<<nb, ENC_NT, 0, s>>>(rho, c.pitch, c.nx, order, n, floor_rho, dx * dy, cum, blk, active);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    enc_blocks_kernel<double><<<1, ENC_NT, 0, s>>>(blk, nb, active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int g = nb < 4096 ? nb : 4096;
    enc_gravity_kernel<T><<<g, ENC_NT, 0, s>>>(order, gend, cum, blk, n, c.nx, c.pitch, x0, y0, dx, dy, cx, cy, G,
                                               soft2, gx, gy, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t EHLaunch<T>::shells(const EHConst<T>& c, const T* rho, const int* order, const int* gend, int n,
                                double* cum, double* blk, const double* geo, double cell_area, double G,
                                double floor_rho, T* gx, T* gy, const int* active, cudaStream_t s) {
    const int nb = (n + ENC_NT - 1) / ENC_NT;
    enc_scan_kernel<T><<<nb, ENC_NT, 0, s>>>(rho, c.pitch, c.nx, order, n, floor_rho, cell_area, cum, blk, active);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    enc_blocks_kernel<double><<<1, ENC_NT, 0, s>>>(blk, nb, active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int g = nb < 4096 ? nb : 4096;
    enc_shell_gravity_kernel<T><<<g, ENC_NT, 0, s>>>(order, gend, cum, blk, geo, n, c.nx, c.pitch, G, gx, gy, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t EHLaunch<T>::speeds(const EHConst<T>& c, const EHFields<T>& st, double* spd_part, double* rho_part,
                                cudaStream_t s) {
    eh_speed_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, st, spd_part, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t EHLaunch<T>::rho_sum(const EHConst<T>& c, const T* rho, double* rho_part, cudaStream_t s) {
    eh_rho_sum_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, rho, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t EHLaunch<T>::diag(const EHConst<T>& c, const EHFields<T>& st, double* part, cudaStream_t s) {
    eh_diag_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, st, part);
    return cudaGetLastError();
}

template <class T>
cudaError_t EHLaunch<T>::derived(const EHConst<T>& c, const EHFields<T>& st, double* out, cudaStream_t s) {
    size_t g = ((size_t)c.nx * c.ny + 255) / 256;
    if (g > 4096) g = 4096;
    eh_derived_kernel<T><<<(int)g, 256, 0, s>>>(c, st, out);
    return cudaGetLastError();
}

}  // namespace ccb
