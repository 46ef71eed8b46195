// Host-side launchers of the 2D Euler/HLLC kernels, defined once per precision
// in euler2d_f64.cu (-fmad=false, the parity path) and euler2d_f32.cu.
#pragma once
#include <cuda_runtime.h>

#include "enclosed_kernels.cuh"
#include "euler2d_kernels.cuh"
#include "mhd2d_launch.h"

namespace ccb {

template <class T> struct EHLaunch {
    static cudaError_t prepare();
    // stage 1: out = floors(in + dt rhs(in)); stage 2: out = floors(0.5 un + 0.5 (in + dt rhs(in)))
    // gravity: gxa/gya (pitched arrays) when non-null, else the centred gradient of phi
    static cudaError_t stage(const EHConst<T>& c, const EHFields<T>& un, const EHFields<T>& in,
                             const EHFields<T>& out, bool stage2, const T* phi, const T* gxa, const T* gya,
                             const double* dt, const int* active, cudaStream_t s);
    // enclosed-mass gravity (enclosed_kernels.cuh) of rho into gx, gy; order / gend: the
    // cells in radius order and each one's group end (host set-up), cum n doubles,
    // blk ceil(n / ENC_NT) doubles of scratch
    static cudaError_t enclosed(const EHConst<T>& c, const T* rho, const int* order, const int* gend, int n,
                                double* cum, double* blk, double x0, double y0, double dx, double dy, double cx,
                                double cy, double G, double soft2, double floor_rho, T* gx, T* gy, const int* active,
                                cudaStream_t s);
    // shell-binned enclosed-mass gravity: order / gend by shell, geo the sorted
    // cells' rx, ry and (r^2 + softening^2)^(3/2) (3 n doubles)
    static cudaError_t shells(const EHConst<T>& c, const T* rho, const int* order, const int* gend, int n, double* cum,
                              double* blk, const double* geo, double cell_area, double G, double floor_rho, T* gx,
                              T* gy, const int* active, cudaStream_t s);
    static cudaError_t speeds(const EHConst<T>& c, const EHFields<T>& st, double* spd_part, double* rho_part,
                              cudaStream_t s);
    static cudaError_t rho_sum(const EHConst<T>& c, const T* rho, double* rho_part, cudaStream_t s);
    static cudaError_t diag(const EHConst<T>& c, const EHFields<T>& st, double* part, cudaStream_t s);
    // rho, P, Mach of the reference's snapshot store, out: 3 planes of nx*ny doubles
    static cudaError_t derived(const EHConst<T>& c, const EHFields<T>& st, double* out, cudaStream_t s);
};

}  // namespace ccb
