// Definitions of M2Launch<T>; included once per precision TU.
#pragma once
#include "mhd2d_launch.h"

namespace ccb {

namespace {
// columns per CTA of the FP32 column pass: at most 256 threads and 48 KB of
// lines (four CTAs per SM)
inline int fft32_cw(int ny) {
    const int tl = fft32_tpl(ny);
    const size_t line = sizeof(float2) * (size_t)fft32_line(ny);
    int cw = 16;
    while (cw > 1 && (cw * tl > 256 || cw * line > 48 * 1024)) cw >>= 1;
    return cw;
}
inline int round32(int t) { return (t + 31) / 32 * 32; }

inline int grid_for(size_t n, int nt, int cap) {
    size_t g = (n + nt - 1) / nt;
    if (g < 1) g = 1;
    if (g > (size_t)cap) g = cap;
    return (int)g;
}
}  // namespace

template <class T>
cudaError_t M2Launch<T>::prepare(int nx, int ny) {
    const int smem = (int)m2_stage_smem<T>();
    cudaError_t e;
#define CC_ATTR(K, BYTES)                                                                              \
    if ((e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (BYTES))) != cudaSuccess) \
        return e;
    CC_ATTR((m2_stage_kernel<T, false, GRAV_NONE>), smem)
    CC_ATTR((m2_stage_kernel<T, false, GRAV_ARRAYS>), smem)
    CC_ATTR((m2_stage_kernel<T, false, GRAV_PHI>), smem)
    CC_ATTR((m2_stage_kernel<T, true, GRAV_NONE>), smem)
    CC_ATTR((m2_stage_kernel<T, true, GRAV_ARRAYS>), smem)
    CC_ATTR((m2_stage_kernel<T, true, GRAV_PHI>), smem)
    if constexpr (sizeof(T) == 4) {
        const int sm0 = (int)MarchG32::smem(false), sm1 = (int)MarchG32::smem(true);
#define CC_MARCH_ATTR(D, G)                                                  \
        CC_ATTR((m2_march_kernel<T, MARCH_W, MARCH_R, D, G, false>), sm0) \
        CC_ATTR((m2_march_kernel<T, MARCH_W, MARCH_R, D, G, true>), sm1)
        CC_MARCH_ATTR(false, GRAV_NONE)
        CC_MARCH_ATTR(false, GRAV_ARRAYS)
        CC_MARCH_ATTR(false, GRAV_PHI)
        CC_MARCH_ATTR(true, GRAV_NONE)
        CC_MARCH_ATTR(true, GRAV_ARRAYS)
        CC_MARCH_ATTR(true, GRAV_PHI)
#undef CC_MARCH_ATTR
        const int smem_c = smem + (int)kahan_smem_extra<T>(StageGeom<T>::NC);
        CC_ATTR((m2_stage_comp_kernel<T, false, GRAV_NONE>), smem_c)
        CC_ATTR((m2_stage_comp_kernel<T, false, GRAV_ARRAYS>), smem_c)
        CC_ATTR((m2_stage_comp_kernel<T, false, GRAV_PHI>), smem_c)
        CC_ATTR((m2_stage_comp_kernel<T, true, GRAV_NONE>), smem_c)
        CC_ATTR((m2_stage_comp_kernel<T, true, GRAV_ARRAYS>), smem_c)
        CC_ATTR((m2_stage_comp_kernel<T, true, GRAV_PHI>), smem_c)
    }
    if constexpr (sizeof(T) == 4) {
        if (nx >= 2 && ny >= 2) {
            const int row = (int)(sizeof(float2) * (size_t)fft32_line(nx));
            const int col = (int)(sizeof(float2) * (size_t)fft32_line(ny)) * fft32_cw(ny);
            if (row <= 227 * 1024 && col <= 227 * 1024) {
                CC_ATTR((f32_rows_fwd_kernel<T, false>), row)
                CC_ATTR((f32_rows_fwd_kernel<T, true>), row)
                CC_ATTR((f32_rows_inv_kernel<T, 0>), row)
                CC_ATTR((f32_rows_inv_kernel<T, 2>), row)
                CC_ATTR((f32_rows_inv_kernel<T, 4>), row)
                CC_ATTR((f32_rows_inv_kernel<T, 8>), row)
                CC_ATTR((f32_rows_inv_kernel<T, 16>), row)
                CC_ATTR((f32_cols_rk_kernel<16, 16>), col)
                CC_ATTR((f32_cols_rk_kernel<8, 2>), col)
                CC_ATTR((f32_cols_rk_kernel<4, 4>), col)
                CC_ATTR((f32_cols_rk_kernel<2, 8>), col)
                CC_ATTR((f32_cols_rk_kernel<1, 16>), col)
                CC_ATTR((f32_cols_rk_kernel<1, 2>), col)
                if (ny >= 256) {
                    const int tsm = (int)fft32_cols_tma_smem(fft32_cw(ny), ny);
                    if (tsm <= 227 * 1024) {
                        CC_ATTR((f32_cols_tma_kernel<16, 16>), tsm)
                        CC_ATTR((f32_cols_tma_kernel<8, 2>), tsm)
                        CC_ATTR((f32_cols_tma_kernel<4, 4>), tsm)
                        CC_ATTR((f32_cols_tma_kernel<2, 8>), tsm)
                        CC_ATTR((f32_cols_tma_kernel<1, 16>), tsm)
                        CC_ATTR((f32_cols_tma_kernel<1, 2>), tsm)
                    }
                }
                CC_ATTR(f32_cols_solve_kernel<1>, col)
                CC_ATTR(f32_cols_solve_kernel<2>, col)
                CC_ATTR(f32_cols_solve_kernel<4>, col)
                CC_ATTR(f32_cols_solve_kernel<8>, col)
                CC_ATTR(f32_cols_solve_kernel<16>, col)
            }
        }
    }
    constexpr int CW = (sizeof(T) == 8) ? 2 : 4;
    const int smem_row = (int)(sizeof(Cplx<T>) * (size_t)fft_line_slots(nx));
    const int smem_col = (int)(sizeof(Cplx<T>) * (size_t)fft_line_slots(ny) * CW);
    if (smem_row <= 227 * 1024 && smem_col <= 227 * 1024) {  // larger lines are rejected by the solver set-up
        CC_ATTR(fft_rows_fwd_kernel<T>, smem_row)
        CC_ATTR(fft_rows_inv_kernel<T>, smem_row)
        CC_ATTR((fft_cols_solve_kernel<T, CW>), smem_col)
    }
#undef CC_ATTR
    return cudaSuccess;
}

template <class T>
cudaError_t M2Launch<T>::stage(const M2Const<T>& c, const Fields<T>& in, const Fields<T>& out, bool defer, int gmode,
                               const T* ga, const T* gb, const double* dt, const int* active, cudaStream_t s) {
    const size_t smem = m2_stage_smem<T>();
    using Gm = StageGeom<T>;
    dim3 grid((c.nx + Gm::TX - 1) / Gm::TX, (c.ny + Gm::TY - 1) / Gm::TY);
#define CC_STAGE_CASE(D, G)                                                                 \
    if (defer == D && gmode == G) {                                                         \
        m2_stage_kernel<T, D, G><<<grid, Gm::NT, smem, s>>>(c, in, out, ga, gb, dt, active); \
        return cudaGetLastError();                                                          \
    }
    CC_STAGE_CASE(false, GRAV_NONE)
    CC_STAGE_CASE(false, GRAV_ARRAYS)
    CC_STAGE_CASE(false, GRAV_PHI)
    CC_STAGE_CASE(true, GRAV_NONE)
    CC_STAGE_CASE(true, GRAV_ARRAYS)
    CC_STAGE_CASE(true, GRAV_PHI)
#undef CC_STAGE_CASE
    return cudaErrorInvalidValue;
}

template <class T>
cudaError_t M2Launch<T>::average(const M2Const<T>& c, const Fields<T>& un, const Fields<T>& s2, const Fields<T>& out,
                                 const double* dt, const int* active, double* spd_part, double* rho_part,
                                 cudaStream_t s) {
    m2_average_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, un, s2, out, dt, active, spd_part, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::stage_comp(const M2Const<T>& c, const Fields<T>& in, const Fields<T>& out,
                                    const Fields<T>& lin, const Fields<T>& lout, bool defer, int gmode, const T* ga,
                                    const T* gb, const double* dt, const int* active, cudaStream_t s) {
    if constexpr (sizeof(T) != 4) {
        return cudaErrorNotSupported;
    } else {
        using Gm = StageGeom<T>;
        const size_t smem = m2_stage_smem<T>() + kahan_smem_extra<T>(Gm::NC);
        dim3 grid((c.nx + Gm::TX - 1) / Gm::TX, (c.ny + Gm::TY - 1) / Gm::TY);
#define CC_STAGE_CASE(D, G)                                                                                  \
        if (defer == D && gmode == G) {                                                                      \
            m2_stage_comp_kernel<T, D, G><<<grid, Gm::NT, smem, s>>>(c, in, out, lin, lout, ga, gb, dt, active); \
            return cudaGetLastError();                                                                       \
        }
        CC_STAGE_CASE(false, GRAV_NONE)
        CC_STAGE_CASE(false, GRAV_ARRAYS)
        CC_STAGE_CASE(false, GRAV_PHI)
        CC_STAGE_CASE(true, GRAV_NONE)
        CC_STAGE_CASE(true, GRAV_ARRAYS)
        CC_STAGE_CASE(true, GRAV_PHI)
#undef CC_STAGE_CASE
        return cudaErrorInvalidValue;
    }
}

template <class T>
cudaError_t M2Launch<T>::stage_march(const M2Const<T>& c, const Fields<T>& in, const Fields<T>& out,
                                     const Fields<T>* lin, const Fields<T>* lout, bool defer, int gmode,
                                     const T* ga, const T* gb, const double* dt, const int* active, int seg_rows,
                                     cudaStream_t s) {
    if constexpr (sizeof(T) != 4) {
        return cudaErrorNotSupported;
    } else {
        if (seg_rows < 1) return cudaErrorInvalidValue;
        const bool kahan = lin && lout;
        const Fields<T> li = kahan ? *lin : Fields<T>{}, lo = kahan ? *lout : Fields<T>{};
        const dim3 grid((c.nx + MARCH_W - 1) / MARCH_W, (c.ny + seg_rows - 1) / seg_rows);
        const size_t smem = MarchG32::smem(kahan);
#define CC_MARCH_CASE(D, G)                                                                                   \
        if (defer == D && gmode == G) {                                                                       \
            if (kahan)                                                                                        \
                m2_march_kernel<T, MARCH_W, MARCH_R, D, G, true><<<grid, MarchG32::NT, smem, s>>>(           \
                    c, in, out, li, lo, ga, gb, dt, active, seg_rows);                                        \
            else                                                                                              \
                m2_march_kernel<T, MARCH_W, MARCH_R, D, G, false><<<grid, MarchG32::NT, smem, s>>>(          \
                    c, in, out, li, lo, ga, gb, dt, active, seg_rows);                                        \
            return cudaGetLastError();                                                                        \
        }
        CC_MARCH_CASE(false, GRAV_NONE)
        CC_MARCH_CASE(false, GRAV_ARRAYS)
        CC_MARCH_CASE(false, GRAV_PHI)
        CC_MARCH_CASE(true, GRAV_NONE)
        CC_MARCH_CASE(true, GRAV_ARRAYS)
        CC_MARCH_CASE(true, GRAV_PHI)
#undef CC_MARCH_CASE
        return cudaErrorInvalidValue;
    }
}

template <class T>
cudaError_t M2Launch<T>::average_comp(const M2Const<T>& c, const Fields<T>& un, const Fields<T>& s2,
                                      const Fields<T>& out, const Fields<T>& unl, const Fields<T>& s2l,
                                      const Fields<T>& outl, const double* dt, const int* active, double* spd_part,
                                      double* rho_part, cudaStream_t s) {
    if constexpr (sizeof(T) != 4) {
        return cudaErrorNotSupported;
    } else {
        m2_average_comp_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, un, s2, out, unl, s2l, outl, dt, active,
                                                                       spd_part, rho_part);
        return cudaGetLastError();
    }
}

template <class T>
cudaError_t M2Launch<T>::speeds(const M2Const<T>& c, const Fields<T>& st, double* spd_part, double* rho_part,
                                cudaStream_t s) {
    m2_speed_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, st, spd_part, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::rho_sum(const M2Const<T>& c, const T* rho, double* rho_part, cudaStream_t s) {
    m2_rho_sum_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, rho, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::diag(const M2Const<T>& c, const Fields<T>& st, double* part, cudaStream_t s) {
    m2_diag_kernel<T, RED_NT><<<RED_BLOCKS, RED_NT, 0, s>>>(c, st, part);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::derived(const M2Const<T>& c, const Fields<T>& st, double* out, cudaStream_t s) {
    m2_derived_kernel<T><<<grid_for((size_t)c.nx * c.ny, 256, 4096), 256, 0, s>>>(c, st, out);
    return cudaGetLastError();
}

// grid of the pack kernels: columns in 256-thread blocks, rows up to 65535
inline dim3 pack_grid(int w, int h) {
    const unsigned gx = (unsigned)((w + 255) / 256);
    const unsigned gy = (unsigned)(h < 65535 ? (h < 1 ? 1 : h) : 65535);
    return dim3(gx < 1 ? 1 : gx, gy);
}

template <class T>
cudaError_t M2Launch<T>::pack_in(const double* src, T* dst, int w, int h, int pitch, cudaStream_t s) {
    pack_in_kernel<T><<<pack_grid(w, h), 256, 0, s>>>(src, dst, w, h, pitch);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::pack_out(const T* src, double* dst, int w, int h, int pitch, cudaStream_t s) {
    pack_out_kernel<T><<<pack_grid(w, h), 256, 0, s>>>(src, dst, w, h, pitch);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::pack_in_split(const double* src, T* hi, T* lo, int w, int h, int pitch, cudaStream_t s) {
    pack_in_split_kernel<T><<<pack_grid(w, h), 256, 0, s>>>(src, hi, lo, w, h, pitch);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::pack_out_sum(const T* hi, const T* lo, double* dst, int w, int h, int pitch,
                                      cudaStream_t s) {
    pack_out_sum_kernel<T><<<pack_grid(w, h), 256, 0, s>>>(hi, lo, dst, w, h, pitch);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::fft_solve(const T* rho, int pitch, const double* rho_part, int nx, int ny, int lognx,
                                   int logny, const Cplx<T>* twx_f, const Cplx<T>* twx_i, const Cplx<T>* twy_f,
                                   const Cplx<T>* twy_i, double Lx, double Ly, double G, Cplx<T>* A, T* phi,
                                   const int* active, cudaStream_t s) {
    constexpr int CW = (sizeof(T) == 8) ? 2 : 4;  // 32-byte column strips
    const size_t smem_row = sizeof(Cplx<T>) * (size_t)fft_line_slots(nx);
    const size_t smem_col = sizeof(Cplx<T>) * (size_t)fft_line_slots(ny) * CW;
    cudaError_t e;
    const int nt_row = nx >= 1024 ? 512 : (nx >= 256 ? 256 : 128);
    fft_rows_fwd_kernel<T><<<ny, nt_row, smem_row, s>>>(rho, pitch, rho_part, RED_BLOCKS, (double)nx * (double)ny, A,
                                                         nx, lognx, twx_f, active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int ncolblk = (nx + CW - 1) / CW;
    fft_cols_solve_kernel<T, CW><<<ncolblk, 512, smem_col, s>>>(A, nx, ny, logny, twy_f, twy_i, Lx, Ly, G, active);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    fft_rows_inv_kernel<T><<<ny, nt_row, smem_row, s>>>(A, nx, lognx, twx_i, phi, pitch, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::fft32_solve(const T* rho, int pitch, const double* rho_part, int nx, int ny,
                                     const float2* rootx, const float2* rooty, double Lx, double Ly, double G,
                                     float2* A, T* phi, const int* active, cudaStream_t s, int* err) {
    if constexpr (sizeof(T) != 4) {
        return cudaErrorNotSupported;
    } else {
        if (nx > FFT32_MAXN || ny > FFT32_MAXN || nx < 2 || ny < 2) return cudaErrorInvalidValue;
        const int nhl = fft32_half_lines(nx);
        const size_t row = sizeof(float2) * (size_t)fft32_line(nx);
        const int cw = fft32_cw(ny);
        const size_t col = sizeof(float2) * (size_t)fft32_line(ny) * cw;
        cudaError_t e;
        // register hand-offs where every thread of a row / column CTA is busy
        // (lines of at least 512 / 256 points); the staged forms below that
        const int rt = round32(fft32_tpl(nx));
        const bool reg_rows = nx >= 512;
        if (reg_rows)
            f32_rows_fwd_kernel<T, true><<<ny / 2, rt, row, s>>>(rho, pitch, rho_part, RED_BLOCKS,
                                                                 (double)nx * (double)ny, A, nx, ny, rootx, active);
        else
            f32_rows_fwd_kernel<T, false><<<ny / 2, rt, row, s>>>(rho, pitch, rho_part, RED_BLOCKS,
                                                                  (double)nx * (double)ny, A, nx, ny, rootx, active);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        const int nt = round32(cw * fft32_tpl(ny)), nb = nhl / cw;
        const int rly = fft32_last_radix(ny);
        if (ny >= 256 && nt == cw * fft32_tpl(ny) && err) {
            static int nsm = 0;
            if (nsm == 0) {
                int dev = 0;
                if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
                if ((e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
            }
            const size_t sm = fft32_cols_tma_smem(cw, ny);
            const int per_sm = (cw == 1 && rly == 2) ? 1 : 2;
            const int g = nb < nsm * per_sm ? nb : nsm * per_sm;
            if (cw == 16 && rly == 16) f32_cols_tma_kernel<16, 16><<<g, nt, sm, s>>>(A, nx, ny, rooty, Lx, Ly, G, active, err);
            else if (cw == 8 && rly == 2) f32_cols_tma_kernel<8, 2><<<g, nt, sm, s>>>(A, nx, ny, rooty, Lx, Ly, G, active, err);
            else if (cw == 4 && rly == 4) f32_cols_tma_kernel<4, 4><<<g, nt, sm, s>>>(A, nx, ny, rooty, Lx, Ly, G, active, err);
            else if (cw == 2 && rly == 8) f32_cols_tma_kernel<2, 8><<<g, nt, sm, s>>>(A, nx, ny, rooty, Lx, Ly, G, active, err);
            else if (cw == 1 && rly == 16) f32_cols_tma_kernel<1, 16><<<g, nt, sm, s>>>(A, nx, ny, rooty, Lx, Ly, G, active, err);
            else if (cw == 1 && rly == 2) f32_cols_tma_kernel<1, 2><<<g, nt, sm, s>>>(A, nx, ny, rooty, Lx, Ly, G, active, err);
            else return cudaErrorInvalidConfiguration;
        } else if (ny >= 256 && nt == cw * fft32_tpl(ny)) {
            if (cw == 16 && rly == 16) f32_cols_rk_kernel<16, 16><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active);
            else if (cw == 8 && rly == 2) f32_cols_rk_kernel<8, 2><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active);
            else if (cw == 4 && rly == 4) f32_cols_rk_kernel<4, 4><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active);
            else if (cw == 2 && rly == 8) f32_cols_rk_kernel<2, 8><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active);
            else if (cw == 1 && rly == 16) f32_cols_rk_kernel<1, 16><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active);
            else if (cw == 1 && rly == 2) f32_cols_rk_kernel<1, 2><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active);
            else return cudaErrorInvalidConfiguration;   // no (columns per CTA, last radix) pair for this ny
        } else {
            switch (cw) {
                case 16: f32_cols_solve_kernel<16><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active); break;
                case 8: f32_cols_solve_kernel<8><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active); break;
                case 4: f32_cols_solve_kernel<4><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active); break;
                case 2: f32_cols_solve_kernel<2><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active); break;
                default: f32_cols_solve_kernel<1><<<nb, nt, col, s>>>(A, nx, ny, rooty, Lx, Ly, G, active); break;
            }
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        switch (reg_rows ? fft32_last_radix(nx) : 0) {
            case 16: f32_rows_inv_kernel<T, 16><<<ny / 2, rt, row, s>>>(A, nx, ny, rootx, phi, pitch, active); break;
            case 8: f32_rows_inv_kernel<T, 8><<<ny / 2, rt, row, s>>>(A, nx, ny, rootx, phi, pitch, active); break;
            case 4: f32_rows_inv_kernel<T, 4><<<ny / 2, rt, row, s>>>(A, nx, ny, rootx, phi, pitch, active); break;
            case 2: f32_rows_inv_kernel<T, 2><<<ny / 2, rt, row, s>>>(A, nx, ny, rootx, phi, pitch, active); break;
            default: f32_rows_inv_kernel<T, 0><<<ny / 2, rt, row, s>>>(A, nx, ny, rootx, phi, pitch, active); break;
        }
        return cudaGetLastError();
    }
}

template <class T>
cudaError_t M2Launch<T>::sor_rhs(const T* rho, int nx, int ny, int pitch, const double* rho_part, double fourpiG,
                                 double floor_rho, double* rhs, const int* active, cudaStream_t s) {
    sor_rhs_kernel<T><<<grid_for((size_t)nx * ny, 256, 2048), 256, 0, s>>>(rho, nx, ny, pitch, rho_part, RED_BLOCKS,
                                                                          fourpiG, floor_rho, rhs, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::phi_to_field(const double* phi, int nx, int ny, T* out, int pitch, const int* active,
                                      cudaStream_t s) {
    phi_to_field_kernel<T><<<grid_for((size_t)nx * ny, 256, 2048), 256, 0, s>>>(phi, nx, ny, out, pitch, active);
    return cudaGetLastError();
}

template <class T>
cudaError_t M2Launch<T>::gravity_from_phi(const T* phi, int nx, int ny, int pitch, AxisMap ax, AxisMap ay, T two_dx,
                                          T two_dy, T* gx, T* gy, cudaStream_t s) {
    gravity_from_phi_kernel<T><<<grid_for((size_t)nx * ny, 256, 2048), 256, 0, s>>>(phi, nx, ny, pitch, ax, ay,
                                                                                   two_dx, two_dy, gx, gy);
    return cudaGetLastError();
}

}  // namespace ccb
