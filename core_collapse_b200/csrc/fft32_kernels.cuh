// FP32 spectral Poisson solve (the bulk path of the periodic FFT gravity).
//
// Same three passes and the same spectral kernel as the FP64 solve in
// poisson_kernels.cuh (navier_stokes_2d_hllc_poisson.cpp:285-328), arranged
// for throughput; the differences change only the rounding:
//   * real-to-complex: rows are real, so two rows ride in one complex
//     transform (z = row_a + i row_b) and only the half spectrum kx = 0..nx/2
//     is stored; the column pass works on nx/2 + 1 columns, the inverse row
//     pass rebuilds the other half from Hermitian symmetry.  Half the
//     transforms and half the work-array traffic.
//   * the work array is kx-major, A[kx * ny + y] (nhl = fft32_half_lines(nx)
//     lines of ny), so the column pass reads and writes contiguous lines; a row
//     pair writes / reads 16 contiguous bytes per kx.
//   * Stockham autosort transforms: radix-16 passes (then one radix 8, 4 or 2
//     pass), 16 values per thread in registers, in-place in shared memory with
//     a barrier between the reads and the writes of a pass, so no bit-reversal
//     pass; log16(n) passes instead of log2(n).  Twiddles from a table of the
//     n-th roots W_n^e = exp(-2 pi i e / n) evaluated in FP64 on the host.
//   * shared-memory lines padded by one element per 16 so that the stride-16
//     writes of the first pass hit distinct banks.
#pragma once
#include <cstdint>

#include <cuda_runtime.h>

namespace ccb {

// threads per CTA at most (n / 16 per line): lines of up to 8192 points.  The
// column pass asks for two such CTAs per SM (at most 64 registers), so that
// four 256-thread CTAs (4096-point lines) are resident per SM; the row passes
// keep their registers (fewer spills, they have the other latencies to hide).
constexpr int FFT32_MAXT = 512;
constexpr int FFT32_MAXN = 16 * FFT32_MAXT;

// kx lines of the half-spectrum work array (nx/2 + 1, rounded up to 16)
__host__ __device__ constexpr int fft32_half_lines(int nx) { return ((nx / 2 + 1) + 15) / 16 * 16; }
__host__ __device__ constexpr int fft32_pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int fft32_line(int n) { return fft32_pad(n - 1) + 1; }   // padded line length
// values per thread (16, or n below 16) and threads per line
__host__ __device__ constexpr int fft32_vals(int n) { return n < 16 ? n : 16; }
__host__ __device__ constexpr int fft32_tpl(int n) { return n / fft32_vals(n); }

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 f2sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// x * w (forward) or x * conj(w) (inverse)
template <bool INV> __device__ __forceinline__ float2 f2twiddle(float2 x, float2 w) {
    if (INV) return make_float2(x.x * w.x + x.y * w.y, x.y * w.x - x.x * w.y);
    return make_float2(x.x * w.x - x.y * w.y, x.x * w.y + x.y * w.x);
}

// x * W_16^e (forward, W_16 = exp(-2 pi i / 16)) or x * W_16^-e (inverse), e in [0, 8)
template <bool INV> __device__ __forceinline__ float2 f2w16(float2 x, int e) {
    constexpr float C[8] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                            0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f};
    constexpr float S[8] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f,
                            1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f};
    if (e == 0) return x;
    if (e == 4) return INV ? make_float2(-x.y, x.x) : make_float2(x.y, -x.x);   // * (+i) or * (-i)
    return f2twiddle<INV>(x, make_float2(C[e], -S[e]));
}

// R-point DFT (R = 2, 4, 8, 16) of v[0..R) in registers, natural order in and
// out: bit-reversal permutation, then radix-2 butterflies (every index is a
// compile-time constant once the loops are unrolled).
template <int R, bool INV> __device__ __forceinline__ void f32_dft(float2* v) {
    constexpr int LR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
#pragma unroll
    for (int i = 0; i < R; i++) {
        int j = 0;
#pragma unroll
        for (int b = 0; b < LR; b++) j |= ((i >> b) & 1) << (LR - 1 - b);
        if (i < j) { const float2 t = v[i]; v[i] = v[j]; v[j] = t; }
    }
#pragma unroll
    for (int h = 1; h < R; h <<= 1) {
#pragma unroll
        for (int i = 0; i < R; i += 2 * h) {
#pragma unroll
            for (int k = 0; k < h; k++) {
                const float2 a = v[i + k];
                const float2 b = f2w16<INV>(v[i + k + h], k * (8 / h));
                v[i + k] = f2add(a, b);
                v[i + k + h] = f2sub(a, b);
            }
        }
    }
}

// One radix-R Stockham pass over a line of n values (padded layout), sub-
// transform length Ns before the pass.  tl threads per line (lt its thread,
// act false for the idle threads of a rounded-up block), each with V / R
// butterflies.  Contains two barriers: every thread of the CTA calls it.
template <int R, int V, bool INV>
__device__ __forceinline__ void f32_pass(float2* a, int n, int Ns, const float2* __restrict__ roots, int lt, int tl,
                                         bool act) {
    constexpr int G = V / R;
    const int nb = n / R;
    float2 v[V];
    if (act) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int j = lt + g * tl;
#pragma unroll
            for (int r = 0; r < R; r++) v[g * R + r] = a[fft32_pad(j + r * nb)];
        }
    }
    __syncthreads();
    if (act) {
        const int span = n / (Ns * R);
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int j = lt + g * tl;
            const int k = j & (Ns - 1);
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; r++) v[g * R + r] = f2twiddle<INV>(v[g * R + r], __ldg(&roots[r * k * span]));
            }
            f32_dft<R, INV>(&v[g * R]);
            const int base = (j - k) * R + k;
#pragma unroll
            for (int s = 0; s < R; s++) a[fft32_pad(base + s * Ns)] = v[g * R + s];
        }
    }
    __syncthreads();
}

// Whole transform of one line (unnormalised); uniform over the CTA.
template <bool INV>
__device__ __forceinline__ void f32_fft_line(float2* a, int n, const float2* __restrict__ roots, int lt, bool act) {
    const int tl = fft32_tpl(n);
    if (n >= 16) {
        int Ns = 1;
        while (n / Ns >= 16) {
            f32_pass<16, 16, INV>(a, n, Ns, roots, lt, tl, act);
            Ns *= 16;
        }
        const int rem = n / Ns;
        if (rem == 8) f32_pass<8, 16, INV>(a, n, Ns, roots, lt, tl, act);
        else if (rem == 4) f32_pass<4, 16, INV>(a, n, Ns, roots, lt, tl, act);
        else if (rem == 2) f32_pass<2, 16, INV>(a, n, Ns, roots, lt, tl, act);
    } else if (n == 8) {
        f32_pass<8, 8, INV>(a, n, 1, roots, lt, tl, act);
    } else if (n == 4) {
        f32_pass<4, 4, INV>(a, n, 1, roots, lt, tl, act);
    } else if (n == 2) {
        f32_pass<2, 2, INV>(a, n, 1, roots, lt, tl, act);
    }
}

// ---------------------------------------------------------------------------
// Register hand-offs (lines of n >= 256 points, every thread of the CTA
// active, tl = n / 16 threads per line).  The first pass of the transform
// (radix 16, Ns = 1) reads x[lt + r tl], r < 16: exactly the values a thread
// fetches with coalesced global loads, so it can start from registers.  The
// last pass (radix RL) leaves X[lt + fft32_fmap<RL>(q) tl] in the thread's
// register q: coalesced again, so the last pass can feed the next step (the
// spectral factor, the inverse transform's first pass, the global store)
// from registers.  This removes the staging round trips through shared
// memory and their barriers; the arithmetic, and so every value, is that of
// f32_fft_line.
// ---------------------------------------------------------------------------
template <int RL> __host__ __device__ constexpr int fft32_fmap(int q) { return q / RL + (q % RL) * (16 / RL); }
// radix of the last pass of an n-point transform (16 when n is a power of 16)
__host__ __device__ constexpr int fft32_last_radix(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return (l % 4 == 0) ? 16 : (1 << (l % 4));
}

// One Stockham pass as f32_pass (V = 16), with its input from registers
// (IN_REG: v[g R + r] = x[j + r n / R], j = lt + g tl) and / or its output
// left in registers (OUT_REG: v[g R + s] = X[base + s Ns]).  Barriers: one
// after the shared-memory writes; one between the reads and the writes of an
// in-place pass.  A pass that reads from registers writes without a barrier
// first, so the caller makes sure nobody still reads the line.
template <int R, bool INV, bool IN_REG, bool OUT_REG>
__device__ __forceinline__ void f32_pass_rw(float2* a, float2 (&v)[16], int n, int Ns,
                                            const float2* __restrict__ roots, int lt, int tl) {
    constexpr int G = 16 / R;
    const int nb = n / R;
    if constexpr (!IN_REG) {
#pragma unroll
        for (int g = 0; g < G; g++) {
            const int j = lt + g * tl;
#pragma unroll
            for (int r = 0; r < R; r++) v[g * R + r] = a[fft32_pad(j + r * nb)];
        }
        if constexpr (!OUT_REG) __syncthreads();
    }
    const int span = n / (Ns * R);
#pragma unroll
    for (int g = 0; g < G; g++) {
        const int j = lt + g * tl;
        const int k = j & (Ns - 1);
        if (Ns > 1) {
#pragma unroll
            for (int r = 1; r < R; r++) v[g * R + r] = f2twiddle<INV>(v[g * R + r], __ldg(&roots[r * k * span]));
        }
        f32_dft<R, INV>(&v[g * R]);
        if constexpr (!OUT_REG) {
            const int base = (j - k) * R + k;
#pragma unroll
            for (int s = 0; s < R; s++) a[fft32_pad(base + s * Ns)] = v[g * R + s];
        }
    }
    if constexpr (!OUT_REG) __syncthreads();
}

// Whole transform of a line, ending in registers: v[q] = X[lt + fft32_fmap<RL>(q) tl]
// on exit.  IN_REG: v[r] = x[lt + r tl] on entry, else the line is in shared memory.
// RL = fft32_last_radix(n).
template <int RL, bool INV, bool IN_REG>
__device__ __forceinline__ void f32_fft_regs(float2* a, float2 (&v)[16], int n, const float2* __restrict__ roots,
                                             int lt) {
    const int tl = n / 16;
    int Ns = 1;
    if constexpr (IN_REG) {
        f32_pass_rw<16, INV, true, false>(a, v, n, 1, roots, lt, tl);
        Ns = 16;
    }
    while (n / Ns > RL) {
        f32_pass_rw<16, INV, false, false>(a, v, n, Ns, roots, lt, tl);
        Ns *= 16;
    }
    f32_pass_rw<RL, INV, false, true>(a, v, n, Ns, roots, lt, tl);
}

// Whole transform of a line from registers (v[r] = x[lt + r tl]) into shared
// memory (natural order), the rest as f32_fft_line.
template <bool INV>
__device__ __forceinline__ void f32_fft_from_regs(float2* a, float2 (&v)[16], int n, const float2* __restrict__ roots,
                                                  int lt) {
    const int tl = n / 16;
    f32_pass_rw<16, INV, true, false>(a, v, n, 1, roots, lt, tl);
    int Ns = 16;
    while (n / Ns >= 16) {
        f32_pass<16, 16, INV>(a, n, Ns, roots, lt, tl, true);
        Ns *= 16;
    }
    const int rem = n / Ns;
    if (rem == 8) f32_pass<8, 16, INV>(a, n, Ns, roots, lt, tl, true);
    else if (rem == 4) f32_pass<4, 16, INV>(a, n, Ns, roots, lt, tl, true);
    else if (rem == 2) f32_pass<2, 16, INV>(a, n, Ns, roots, lt, tl, true);
}

// pass 1: rows 2b and 2b+1 -> half spectra.  rho pitched; mean = sum/N.
// REG: the first pass starts from the loaded registers (blockDim = nx / 16).
template <class F, bool REG>   // F = float (a template so that only the FP32 unit instantiates it)
__global__ void __maxnreg__(80)   // three 256-thread CTAs per SM; blocks of up to FFT32_MAXT threads
f32_rows_fwd_kernel(const F* __restrict__ rho, int pitch, const double* __restrict__ rho_part, int nparts,
                    double ncell, float2* __restrict__ A, int nx, int ny, const float2* __restrict__ roots,
                    const int* __restrict__ active) {
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* a = reinterpret_cast<float2*>(smem_raw);
    __shared__ double s_mean;
    const int ja = 2 * blockIdx.x, jb = ja + 1;
    // the two rows into registers first (at most 16 values per thread:
    // blockDim >= nx / 16), so their loads are in flight while warp 0 forms
    // the mean from the density partials (lane-strided sums, shuffle tree)
    float ra[16], rb[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int i = threadIdx.x + q * blockDim.x;
        if (i < nx) { ra[q] = rho[(size_t)ja * pitch + i]; rb[q] = rho[(size_t)jb * pitch + i]; }
    }
    if (threadIdx.x < 32) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nparts; b += 32) s += rho_part[b];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) s_mean = s / ncell;
    }
    __syncthreads();
    const float mean = (float)s_mean;
    if constexpr (REG) {
        float2 v[16];
#pragma unroll
        for (int q = 0; q < 16; q++) v[q] = make_float2(ra[q] - mean, rb[q] - mean);
        f32_fft_from_regs<false>(a, v, nx, roots, (int)threadIdx.x);
    } else {
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int i = threadIdx.x + q * blockDim.x;
            if (i < nx) a[fft32_pad(i)] = make_float2(ra[q] - mean, rb[q] - mean);
        }
        __syncthreads();
        const int tl = fft32_tpl(nx);
        f32_fft_line<false>(a, nx, roots, (int)threadIdx.x, (int)threadIdx.x < tl);
    }
    // Z = FFT(x_a + i x_b):  X_a[k] = (Z[k] + conj Z[-k]) / 2,  X_b[k] = (Z[k] - conj Z[-k]) / (2 i)
    for (int k = threadIdx.x; k <= nx / 2; k += blockDim.x) {
        const float2 z = a[fft32_pad(k)], m = a[fft32_pad((nx - k) & (nx - 1))];
        *reinterpret_cast<float4*>(A + (size_t)k * ny + ja) =
            make_float4(0.5f * (z.x + m.x), 0.5f * (z.y - m.y), 0.5f * (z.y + m.y), 0.5f * (m.x - z.x));
    }
}

// pass 2: CW columns kx = c0 .. c0+CW-1 (those <= nx/2): forward FFT along y,
// spectral kernel, inverse FFT along y, 1/ny.
template <int CW>
__global__ void __launch_bounds__(FFT32_MAXT, 2)
f32_cols_solve_kernel(float2* __restrict__ A, int nx, int ny, const float2* __restrict__ roots, double Lx, double Ly,
                      double G, const int* __restrict__ active) {
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* a = reinterpret_cast<float2*>(smem_raw);
    const int LP = fft32_line(ny);
    const int c0 = blockIdx.x * CW;
    const int ncol = nx / 2 + 1;
    // all of this thread's values in flight before any is stored (at most 16
    // per thread: blockDim >= CW ny / 16); ny is a power of two
    const int lgy = __ffs(ny) - 1;
    float2 xr[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = threadIdx.x + q * blockDim.x, cc = k >> lgy;
        xr[q] = (k < CW * ny && c0 + cc < ncol) ? A[(size_t)c0 * ny + k] : make_float2(0.0f, 0.0f);
    }
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int k = threadIdx.x + q * blockDim.x;
        if (k < CW * ny) a[(k >> lgy) * LP + fft32_pad(k & (ny - 1))] = xr[q];
    }
    __syncthreads();
    const int tl = fft32_tpl(ny);
    const int l = (int)threadIdx.x / tl, lt = (int)threadIdx.x % tl;
    const bool act = l < CW;
    float2* line = a + (act ? l : 0) * LP;
    f32_fft_line<false>(line, ny, roots, lt, act);
    // spectral kernel (NS:308-322), continuous |k|^2, zero mode removed; in
    // FP32 here (the factor carries the FP32 solve's rounding anyway)
    const float fy = (float)(2.0 * M_PI / Ly), fx = (float)(2.0 * M_PI / Lx), g4 = (float)(4.0 * M_PI * G);
    for (int k = threadIdx.x; k < CW * ny; k += blockDim.x) {
        const int cc = k / ny, j = k % ny, i = c0 + cc;
        const int nj = (j <= ny / 2) ? j : j - ny;
        const float ky = fy * (float)nj, kx = fx * (float)i;
        const float k2 = kx * kx + ky * ky;
        float2& z = a[cc * LP + fft32_pad(j)];
        if (k2 == 0.0f) {
            z = make_float2(0.0f, 0.0f);
        } else {
            const float s = -g4 / k2;
            z.x = z.x * s;
            z.y = z.y * s;
        }
    }
    __syncthreads();
    f32_fft_line<true>(line, ny, roots, lt, act);
    const float n = (float)ny;
    for (int k = threadIdx.x; k < CW * ny; k += blockDim.x) {
        const int cc = k / ny, j = k % ny;
        if (c0 + cc >= ncol) continue;
        const float2 z = a[cc * LP + fft32_pad(j)];
        A[(size_t)(c0 + cc) * ny + j] = make_float2(z.x / n, z.y / n);
    }
}

// pass 2 with register hand-offs (ny >= 256, blockDim = CW ny / 16): the
// column's values go from global loads into the forward transform's first
// pass, the forward transform's last pass hands its registers to the spectral
// factor and on to the inverse transform's first pass, and the inverse's last
// pass stores from registers (coalesced).  RL = fft32_last_radix(ny).
// Two 256-thread CTAs per SM (up to 128 registers): the 16 values of a line
// stay live across the hand-offs; at three CTAs (80 registers) they spill and
// the pass is slower (4096^2 step 3.534 against 3.555 ms).
template <int CW, int RL>
__global__ void __launch_bounds__(CW == 1 && RL == 2 ? 512 : 256, CW == 1 && RL == 2 ? 1 : 2)
f32_cols_rk_kernel(float2* __restrict__ A, int nx, int ny, const float2* __restrict__ roots, double Lx, double Ly,
                   double G, const int* __restrict__ active) {
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* a = reinterpret_cast<float2*>(smem_raw);
    const int tl = ny / 16;
    const int l = (int)threadIdx.x / tl, lt = (int)threadIdx.x % tl;
    const int kx = blockIdx.x * CW + l;
    const bool live = kx < nx / 2 + 1;
    float2* line = a + l * fft32_line(ny);
    float2* col = A + (size_t)kx * ny;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; r++) v[r] = live ? col[lt + r * tl] : make_float2(0.0f, 0.0f);
    f32_fft_regs<RL, false, true>(line, v, ny, roots, lt);
    // spectral kernel (NS:308-322) on the registers, as in f32_cols_solve_kernel
    const float fy = (float)(2.0 * M_PI / Ly), fx = (float)(2.0 * M_PI / Lx), g4 = (float)(4.0 * M_PI * G);
    float2 w[16];
#pragma unroll
    for (int q = 0; q < 16; q++) {
        const int j = lt + fft32_fmap<RL>(q) * tl;
        const int nj = (j <= ny / 2) ? j : j - ny;
        const float ky = fy * (float)nj, kxf = fx * (float)kx;
        const float k2 = kxf * kxf + ky * ky;
        float2 z = v[q];
        if (k2 == 0.0f) {
            z = make_float2(0.0f, 0.0f);
        } else {
            const float sf = -g4 / k2;
            z.x = z.x * sf;
            z.y = z.y * sf;
        }
        w[fft32_fmap<RL>(q)] = z;   // the inverse's first-pass order: w[r] = Z[lt + r tl]
    }
    __syncthreads();   // every thread's last forward reads of the line are done
    f32_fft_regs<RL, true, true>(line, w, ny, roots, lt);
    if (live) {
        const float n = (float)ny;
#pragma unroll
        for (int q = 0; q < 16; q++) col[lt + fft32_fmap<RL>(q) * tl] = make_float2(w[q].x / n, w[q].y / n);
    }
}

// ---------------------------------------------------------------------------
// Bulk-copy (TMA) staging for the column pass.  A line group (CW contiguous kx
// lines, CW ny float2, 16-byte aligned, a multiple of 16 bytes) is one
// cp.async.bulk copy from global into shared memory, completed on an
// mbarrier with its byte count; no multicast, this GPU's memory only.  Every
// wait is bounded: after FFT32_WAIT_POLLS polls the kernel records the timeout
// in *err, waits (bounded again) for its copies still in flight and returns.
// ---------------------------------------------------------------------------
constexpr unsigned FFT32_WAIT_POLLS = 1u << 22;

__device__ __forceinline__ uint32_t f32_smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void f32_mbar_init(uint32_t mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
}
// one elected thread: expect `bytes` on the mbarrier and start the copy
__device__ __forceinline__ void f32_bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // earlier generic reads of dst come first
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mbar)
                 : "memory");
}
// true once phase `parity` of the mbarrier has completed; false after the poll limit
__device__ __forceinline__ bool f32_mbar_wait(uint32_t mbar, uint32_t parity) {
    for (unsigned it = 0; it < FFT32_WAIT_POLLS; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        __nanosleep(32);
    }
    return false;
}

// shared memory of f32_cols_tma_kernel: two staging buffers, the padded work
// lines, two mbarriers
__host__ __device__ constexpr size_t fft32_cols_tma_smem(int cw, int ny) {
    return sizeof(float2) * (2 * (size_t)cw * ny + (size_t)cw * fft32_line(ny)) + 16;
}

// Pass 2 as f32_cols_rk_kernel, persistent: a CTA takes line groups
// blockIdx.x, blockIdx.x + gridDim.x, ...; while it transforms one group the
// bulk copy of its next group is in flight into the other staging buffer, so
// the global load latency of the column pass is hidden behind the transform.
// The first forward pass reads the staged line (coalesced shared loads); the
// rest, and every value, is f32_cols_rk_kernel's.
template <int CW, int RL>
__global__ void __launch_bounds__(CW == 1 && RL == 2 ? 512 : 256, CW == 1 && RL == 2 ? 1 : 2)
f32_cols_tma_kernel(float2* __restrict__ A, int nx, int ny, const float2* __restrict__ roots, double Lx, double Ly,
                    double G, const int* __restrict__ active, int* __restrict__ err) {
    if (active && *active == 0) return;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    const int tl = ny / 16;
    const int l = (int)threadIdx.x / tl, lt = (int)threadIdx.x % tl;
    const int ncol = nx / 2 + 1, ngroups = (ncol + CW - 1) / CW;
    const int gsz = CW * ny;                                   // float2 per group
    float2* stage = reinterpret_cast<float2*>(smem_raw);       // 2 x gsz
    float2* work = stage + 2 * gsz;                            // CW padded lines
    uint64_t* mbar = reinterpret_cast<uint64_t*>(work + CW * fft32_line(ny));
    const uint32_t mb[2] = {f32_smem_addr(&mbar[0]), f32_smem_addr(&mbar[1])};
    const uint32_t st[2] = {f32_smem_addr(stage), f32_smem_addr(stage + gsz)};
    const uint32_t bytes = (uint32_t)(sizeof(float2) * gsz);
    if (threadIdx.x == 0) {
        f32_mbar_init(mb[0]);
        f32_mbar_init(mb[1]);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    int g = blockIdx.x;
    if (threadIdx.x == 0 && g < ngroups) f32_bulk_load(st[0], A + (size_t)g * gsz, bytes, mb[0]);
    const float fy = (float)(2.0 * M_PI / Ly), fx = (float)(2.0 * M_PI / Lx), g4 = (float)(4.0 * M_PI * G);
    float2* line = work + l * fft32_line(ny);
    for (int it = 0; g < ngroups; g += gridDim.x, ++it) {
        const int buf = it & 1;
        const bool next = g + (int)gridDim.x < ngroups;
        if (threadIdx.x == 0 && next)
            f32_bulk_load(st[buf ^ 1], A + (size_t)(g + gridDim.x) * gsz, bytes, mb[buf ^ 1]);
        const bool ok = f32_mbar_wait(mb[buf], (it >> 1) & 1);
        if (!__syncthreads_and(ok)) {
            if (threadIdx.x == 0) {
                atomicExch(err, 1);
                f32_mbar_wait(mb[buf], (it >> 1) & 1);                   // let the copies in flight land
                if (next) f32_mbar_wait(mb[buf ^ 1], ((it + 1) >> 1) & 1);
            }
            __syncthreads();
            return;
        }
        const float2* src = stage + buf * gsz + l * ny;
        float2 v[16];
#pragma unroll
        for (int r = 0; r < 16; r++) v[r] = src[lt + r * tl];
        const int kx = g * CW + l;
        f32_fft_regs<RL, false, true>(line, v, ny, roots, lt);
        float2 w[16];
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int j = lt + fft32_fmap<RL>(q) * tl;
            const int nj = (j <= ny / 2) ? j : j - ny;
            const float ky = fy * (float)nj, kxf = fx * (float)kx;
            const float k2 = kxf * kxf + ky * ky;
            float2 z = v[q];
            if (k2 == 0.0f) {
                z = make_float2(0.0f, 0.0f);
            } else {
                const float sf = -g4 / k2;
                z.x = z.x * sf;
                z.y = z.y * sf;
            }
            w[fft32_fmap<RL>(q)] = z;
        }
        __syncthreads();   // every thread's last forward reads of the line are done
        f32_fft_regs<RL, true, true>(line, w, ny, roots, lt);
        if (kx < ncol) {
            float2* col = A + (size_t)kx * ny;
            const float n = (float)ny;
#pragma unroll
            for (int q = 0; q < 16; q++) col[lt + fft32_fmap<RL>(q) * tl] = make_float2(w[q].x / n, w[q].y / n);
        }
        __syncthreads();   // the line's last reads are done before the next group's first pass writes it
    }
}

// pass 3: half spectra of rows 2b, 2b+1 -> Z = X_a + i X_b over all kx
// (Hermitian completion), inverse FFT, phi_a = Re / nx, phi_b = Im / nx.
// RL > 0: the last pass stores phi from registers (blockDim = nx / 16,
// RL = fft32_last_radix(nx)).
template <class F, int RL>   // F = float (a template so that only the FP32 unit instantiates it)
__global__ void __launch_bounds__(FFT32_MAXT)
f32_rows_inv_kernel(const float2* __restrict__ A, int nx, int ny, const float2* __restrict__ roots,
                    F* __restrict__ phi, int pitch, const int* __restrict__ active) {
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float2* a = reinterpret_cast<float2*>(smem_raw);
    const int ja = 2 * blockIdx.x, jb = ja + 1;
    // all of this thread's half-spectrum values in flight before any is used
    // (at most 9 per thread: blockDim >= nx / 16)
    float4 xr[9];
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const int k = threadIdx.x + q * blockDim.x;
        if (k <= nx / 2) xr[q] = *reinterpret_cast<const float4*>(A + (size_t)k * ny + ja);
    }
#pragma unroll
    for (int q = 0; q < 9; q++) {
        const int k = threadIdx.x + q * blockDim.x;
        if (k > nx / 2) break;
        const float2 xa = make_float2(xr[q].x, xr[q].y), xb = make_float2(xr[q].z, xr[q].w);
        a[fft32_pad(k)] = make_float2(xa.x - xb.y, xa.y + xb.x);
        if (k > 0 && k < nx / 2) a[fft32_pad(nx - k)] = make_float2(xa.x + xb.y, xb.x - xa.y);
    }
    __syncthreads();
    const float n = (float)nx;
    if constexpr (RL > 0) {
        float2 v[16];
        f32_fft_regs<RL, true, false>(a, v, nx, roots, (int)threadIdx.x);
        const int tl = nx / 16;
#pragma unroll
        for (int q = 0; q < 16; q++) {
            const int i = (int)threadIdx.x + fft32_fmap<RL>(q) * tl;
            phi[(size_t)ja * pitch + i] = v[q].x / n;
            phi[(size_t)jb * pitch + i] = v[q].y / n;
        }
    } else {
        const int tl = fft32_tpl(nx);
        f32_fft_line<true>(a, nx, roots, (int)threadIdx.x, (int)threadIdx.x < tl);
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            const float2 z = a[fft32_pad(i)];
            phi[(size_t)ja * pitch + i] = z.x / n;
            phi[(size_t)jb * pitch + i] = z.y / n;
        }
    }
}

}  // namespace ccb
