// Host-side launchers of the 2D Navier-Stokes kernels, defined once per
// precision in ns2d_f64.cu (-fmad=false, the parity path) and ns2d_f32.cu.
// The spectral Poisson solve is the 2D MHD solver's (M2Launch<T>::fft_solve /
// fft32_solve).
#pragma once
#include <cuda_runtime.h>

#include "mhd2d_launch.h"
#include "ns2d_kernels.cuh"

namespace ccb {

template <class T> struct NSLaunch {
    static cudaError_t prepare();
    // stage 1: k1 = rhs(in), out = in + dt k1; stage 2: out = un + dt/2 (k1 + rhs(in)); rho floored
    static cudaError_t stage(const NSConst<T>& c, const NSFields<T>& un, const NSFields<T>& in,
                             const NSFields<T>& k1, const NSFields<T>& out, bool stage2, const T* phi,
                             const double* dt, const int* active, cudaStream_t s);
    // RED_BLOCKS partials of the CFL speed, the minimum and the sum of the floored density
    static cudaError_t speeds(const NSConst<T>& c, const NSFields<T>& st, double* spd_part, double* rmin_part,
                              double* rho_part, cudaStream_t s);
    static cudaError_t rho_sum(const NSConst<T>& c, const T* d, double* rho_part, cudaStream_t s);
    static cudaError_t floor_copy(const NSConst<T>& c, const T* d, T* out, const int* active, cudaStream_t s);
    static cudaError_t gravity(const NSConst<T>& c, const T* phi, T* gx, T* gy, cudaStream_t s);
    static cudaError_t diag(const NSConst<T>& c, const NSFields<T>& st, double* part, cudaStream_t s);
    // rho, P, Mach, u, v, momx, momy, Phi of the reference's snapshot store, out: 8 planes of nx*ny doubles
    static cudaError_t derived(const NSConst<T>& c, const NSFields<T>& st, const T* phi, double* out, cudaStream_t s);
};

// compute_dt + the loop's clamp to t_end, from the speeds() partials (one thread)
cudaError_t launch_ns_dt(const double* spd_part, const double* rmin_part, NSDtSpec d, double* dt_out,
                         const double* t_now, int* active, cudaStream_t s);

}  // namespace ccb
