// Host-side launchers of the 2D MHD and Poisson kernels.  Defined once per
// precision in mhd2d_f64.cu (built with -fmad=false: the parity path) and
// mhd2d_f32.cu (FMA contraction on: the bulk path).
#pragma once
#include <cuda_runtime.h>

#include "fft32_kernels.cuh"
#include "mhd2d_kernels.cuh"
#include "mhd2d_march.cuh"
#include "poisson_kernels.cuh"

namespace ccb {

constexpr int RED_NT = 512;      // threads of the reduction kernels (two blocks per SM at <= 64 registers)
constexpr int RED_BLOCKS = 296;  // 2 x 148 SMs; fixed so reduction order is fixed

template <class T> struct M2Launch {
    // raise the dynamic shared-memory limits of the kernels (once per device, before any launch or capture)
    static cudaError_t prepare(int nx, int ny);
    static cudaError_t stage(const M2Const<T>& c, const Fields<T>& in, const Fields<T>& out, bool defer, int gmode,
                             const T* ga, const T* gb, const double* dt, const int* active, cudaStream_t s);
    static cudaError_t average(const M2Const<T>& c, const Fields<T>& un, const Fields<T>& s2, const Fields<T>& out,
                               const double* dt, const int* active, double* spd_part, double* rho_part,
                               cudaStream_t s);
    // the same two kernels on compensated states (FP32 only; l*: the residual planes)
    static cudaError_t stage_comp(const M2Const<T>& c, const Fields<T>& in, const Fields<T>& out,
                                  const Fields<T>& lin, const Fields<T>& lout, bool defer, int gmode, const T* ga,
                                  const T* gb, const double* dt, const int* active, cudaStream_t s);
    static cudaError_t average_comp(const M2Const<T>& c, const Fields<T>& un, const Fields<T>& s2,
                                    const Fields<T>& out, const Fields<T>& unl, const Fields<T>& s2l,
                                    const Fields<T>& outl, const double* dt, const int* active, double* spd_part,
                                    double* rho_part, cudaStream_t s);
    // FP32 column-march stage (mhd2d_march.cuh): segments of seg_rows rows;
    // lin / lout non-null: compensated state
    static cudaError_t stage_march(const M2Const<T>& c, const Fields<T>& in, const Fields<T>& out,
                                   const Fields<T>* lin, const Fields<T>* lout, bool defer, int gmode, const T* ga,
                                   const T* gb, const double* dt, const int* active, int seg_rows, cudaStream_t s);
    static cudaError_t pack_in_split(const double* src, T* hi, T* lo, int w, int h, int pitch, cudaStream_t s);
    static cudaError_t pack_out_sum(const T* hi, const T* lo, double* dst, int w, int h, int pitch, cudaStream_t s);
    static cudaError_t speeds(const M2Const<T>& c, const Fields<T>& st, double* spd_part, double* rho_part,
                              cudaStream_t s);
    static cudaError_t rho_sum(const M2Const<T>& c, const T* rho, double* rho_part, cudaStream_t s);
    static cudaError_t diag(const M2Const<T>& c, const Fields<T>& st, double* part, cudaStream_t s);
    // the 10 derived snapshot fields of the reference's store, out: 10 planes of nx*ny doubles
    static cudaError_t derived(const M2Const<T>& c, const Fields<T>& st, double* out, cudaStream_t s);
    static cudaError_t pack_in(const double* src, T* dst, int w, int h, int pitch, cudaStream_t s);
    static cudaError_t pack_out(const T* src, double* dst, int w, int h, int pitch, cudaStream_t s);
    // spectral solve: rho (pitched T) -> phi (pitched T); A: nx*ny complex work
    static cudaError_t fft_solve(const T* rho, int pitch, const double* rho_part, int nx, int ny, int lognx,
                                 int logny, const Cplx<T>* twx_f, const Cplx<T>* twx_i, const Cplx<T>* twy_f,
                                 const Cplx<T>* twy_i, double Lx, double Ly, double G, Cplx<T>* A, T* phi,
                                 const int* active, cudaStream_t s);
    // FP32 spectral solve (fft32_kernels.cuh), T = float only: rootx / rooty
    // the nx-th / ny-th roots of unity W^e = (cos 2 pi e/n, -sin 2 pi e/n),
    // A: fft32_half_lines(nx) x ny complex work array; needs nx, ny powers of two.
    // err (device int): given, the column pass stages its lines by bulk copies
    // (f32_cols_tma_kernel) and records a timed-out copy wait there.
    static cudaError_t fft32_solve(const T* rho, int pitch, const double* rho_part, int nx, int ny,
                                   const float2* rootx, const float2* rooty, double Lx, double Ly, double G,
                                   float2* A, T* phi, const int* active, cudaStream_t s, int* err = nullptr);
    static cudaError_t sor_rhs(const T* rho, int nx, int ny, int pitch, const double* rho_part, double fourpiG,
                               double floor_rho, double* rhs, const int* active, cudaStream_t s);
    static cudaError_t phi_to_field(const double* phi, int nx, int ny, T* out, int pitch, const int* active,
                                    cudaStream_t s);
    static cudaError_t gravity_from_phi(const T* phi, int nx, int ny, int pitch, AxisMap ax, AxisMap ay, T two_dx,
                                        T two_dy, T* gx, T* gy, cudaStream_t s);
};

cudaError_t launch_dt_finalize(const double* spd_part, DtSpec d, double* dt_out, const double* t_now, int* active,
                               cudaStream_t s);
cudaError_t launch_clock(double* t, const double* dt, const int* active, long long* steps, cudaStream_t s);
// cooperative launch of the red-black SOR; nblocks must all be co-resident
cudaError_t launch_sor(const SorArgs& a, int* nblocks_out, cudaStream_t s);
// the lexicographic SOR of the reference (one CTA, sor_lex_kernel); rho pitched
template <class T> cudaError_t launch_sor_lex(const SorLexArgs& a, const T* rho, cudaStream_t s);

}  // namespace ccb
