// Self-gravity Poisson solves (templated on T; instantiated per precision).
//
// Spectral periodic solve (navier_stokes_2d_hllc_poisson.cpp:285-328), three
// passes over a complex work array A (nx*ny, row-major):
//   1. rows:    A = FFT_x(rho - mean)                      (fft_rows_fwd)
//   2. columns: A = IFFT_y( K(k) * FFT_y(A) ),  K = -4 pi G / |k|^2, K(0)=0
//   3. rows:    phi = Re IFFT_x(A)
// Every 1D transform is the reference's radix-2 decimation-in-time FFT
// (NS:152-177): bit-reversed load, log2(n) butterfly passes with twiddles built
// on the host by the reference's recurrence w *= wlen, inverse scaled by 1/n.
// The reference runs the inverse as rows-then-columns; here it is
// columns-then-rows so that the column inverse fuses with the spectral
// multiply (rounding differs at the 1e-16 level; stated in the tests).
//
// Red-black SOR (the GPU ordering of M2:207-223 / EH:335-368): a persistent
// cooperative kernel, one grid barrier per colour, deterministic FP64 mean
// removal after each sweep (applied lazily, see sor_rb_kernel), optional
// residual test.
#pragma once
#include "cc_device.cuh"

namespace ccb {

template <class T> struct Cplx { T re, im; };

// the reference's complex product (x.re*w.re - x.im*w.im, x.re*w.im + x.im*w.re)
template <class T> __device__ __forceinline__ Cplx<T> cmul(Cplx<T> x, Cplx<T> w) {
    Cplx<T> r;
    r.re = x.re * w.re - x.im * w.im;
    r.im = x.re * w.im + x.im * w.re;
    return r;
}

__device__ __forceinline__ int bitrev(int i, int logn) { return (int)(__brev((unsigned)i) >> (32 - logn)); }

// Shared-memory slot of element i of a transform line: one spare slot after
// every 16, so that the strided accesses of the grouped passes below hit
// distinct banks.  A line of n elements takes fft_line_slots(n) slots.
__host__ __device__ constexpr int fft_line_slots(int n) { return n + (n >> 4); }
__device__ __forceinline__ int fpad(int i) { return i + (i >> 4); }

// R consecutive radix-2 stages (half-lengths h0, 2 h0, ..., 2^(R-1) h0) of the
// reference's DIT transform over `lines` lines of n elements in shared memory.
// A thread takes the 2^R elements base + m h0 (m < 2^R) of one group, which
// only exchange data among themselves in these stages, and runs the stages in
// registers: every butterfly u = a[p], v = a[p+h] * tw[h-1 + (p mod h)],
// a[p] = u + v, a[p+h] = u - v is the reference's, with the same operands and
// twiddle, so the result is the same bit for bit as one stage per pass.
template <class T, int R>
__device__ __forceinline__ void fft_group_pass(Cplx<T>* a, int n, int lines, int h0,
                                               const Cplx<T>* __restrict__ tw) {
    constexpr int M = 1 << R;
    const int gpl = n >> R;   // groups per line
    const int L = fft_line_slots(n);
    for (int g = threadIdx.x; g < lines * gpl; g += blockDim.x) {
        const int l = g / gpl, gg = g - l * gpl;
        const int o = gg & (h0 - 1), blk = gg / h0;
        Cplx<T>* line = a + l * L;
        const int base = blk * (M * h0) + o;
        Cplx<T> x[M];
#pragma unroll
        for (int m = 0; m < M; m++) x[m] = line[fpad(base + m * h0)];
#pragma unroll
        for (int st = 0; st < R; st++) {
            const int hs = 1 << st, h = h0 << st;
#pragma unroll
            for (int m = 0; m < M; m++) {
                if (m & hs) continue;
                const Cplx<T> w = tw[h - 1 + o + (m & (hs - 1)) * h0];   // p mod h = o + (m mod hs) h0
                const Cplx<T> u = x[m];
                const Cplx<T> v = cmul(x[m + hs], w);
                x[m].re = u.re + v.re; x[m].im = u.im + v.im;
                x[m + hs].re = u.re - v.re; x[m + hs].im = u.im - v.im;
            }
        }
#pragma unroll
        for (int m = 0; m < M; m++) line[fpad(base + m * h0)] = x[m];
    }
    __syncthreads();
}

// All log2(n) stages over `lines` lines already in bit-reversed order (line l
// at a + l fft_line_slots(n), padded slots), four stages per pass.
// tw: twiddles of all stages, half-length h at tw[h-1 .. 2h-2].
template <class T>
__device__ __forceinline__ void fft_passes(Cplx<T>* a, int n, int lines, const Cplx<T>* __restrict__ tw) {
    int h0 = 1;
    while (h0 < n) {
        const int left = n / h0;
        if (left >= 16) { fft_group_pass<T, 4>(a, n, lines, h0, tw); h0 <<= 4; }
        else if (left == 8) { fft_group_pass<T, 3>(a, n, lines, h0, tw); h0 <<= 3; }
        else if (left == 4) { fft_group_pass<T, 2>(a, n, lines, h0, tw); h0 <<= 2; }
        else { fft_group_pass<T, 1>(a, n, lines, h0, tw); h0 <<= 1; }
    }
}

// the three kernels below run on at most FFT_NT threads
constexpr int FFT_NT = 512;

// pass 1: one block per row.  rho is a pitched T field; mean = sum/N.
template <class T>
__global__ void __launch_bounds__(FFT_NT) fft_rows_fwd_kernel(const T* __restrict__ rho, int pitch, const double* __restrict__ rho_part,
                                    int nparts, double ncell, Cplx<T>* __restrict__ A, int nx, int logn,
                                    const Cplx<T>* __restrict__ tw, const int* __restrict__ active) {
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cplx<T>* a = reinterpret_cast<Cplx<T>*>(smem_raw);
    __shared__ double s_mean;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nparts; b++) s += rho_part[b];
        s_mean = s / ncell;
    }
    __syncthreads();
    const T mean = (T)s_mean;
    const int j = blockIdx.x;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        Cplx<T> z;
        z.re = rho[(size_t)j * pitch + i] - mean;
        z.im = T(0);
        a[fpad(bitrev(i, logn))] = z;
    }
    __syncthreads();
    fft_passes(a, nx, 1, tw);
    for (int i = threadIdx.x; i < nx; i += blockDim.x) A[(size_t)j * nx + i] = a[fpad(i)];
}

// pass 2: CW adjacent columns per block: forward FFT along y, spectral
// multiply, inverse FFT along y.
template <class T, int CW>
__global__ void __launch_bounds__(FFT_NT) fft_cols_solve_kernel(Cplx<T>* __restrict__ A, int nx, int ny, int logn,
                                      const Cplx<T>* __restrict__ twf, const Cplx<T>* __restrict__ twi,
                                      double Lx, double Ly, double G, const int* __restrict__ active) {
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cplx<T>* a = reinterpret_cast<Cplx<T>*>(smem_raw);   // CW padded lines of ny
    const int L = fft_line_slots(ny);
    const int c0 = blockIdx.x * CW;
    for (int k = threadIdx.x; k < CW * ny; k += blockDim.x) {
        const int cc = k % CW, j = k / CW;
        a[cc * L + fpad(bitrev(j, logn))] = A[(size_t)j * nx + c0 + cc];
    }
    __syncthreads();
    fft_passes(a, ny, CW, twf);
    // spectral kernel (NS:308-322), continuous |k|^2, zero mode removed
    const double two_pi = 2.0 * M_PI;
    for (int k = threadIdx.x; k < CW * ny; k += blockDim.x) {
        const int cc = k % CW, j = k / CW, i = c0 + cc;
        const int nj = (j <= ny / 2) ? j : j - ny;
        const int ni = (i <= nx / 2) ? i : i - nx;
        const double ky = two_pi * (double)nj / Ly;
        const double kx = two_pi * (double)ni / Lx;
        const double k2 = kx * kx + ky * ky;
        Cplx<T>& z = a[cc * L + fpad(j)];
        if (k2 == 0.0) { z.re = T(0); z.im = T(0); }
        else {
            const T s = (T)(-(4.0 * M_PI * G) / k2);
            z.re = z.re * s; z.im = z.im * s;
        }
    }
    __syncthreads();
    // bit-reverse permutation of each line for the inverse DIT transform
    for (int k = threadIdx.x; k < CW * ny; k += blockDim.x) {
        const int cc = k / ny, j = k % ny, r = bitrev(j, logn);
        if (j < r) {
            Cplx<T> t = a[cc * L + fpad(j)];
            a[cc * L + fpad(j)] = a[cc * L + fpad(r)];
            a[cc * L + fpad(r)] = t;
        }
    }
    __syncthreads();
    fft_passes(a, ny, CW, twi);
    const T n = (T)ny;
    for (int k = threadIdx.x; k < CW * ny; k += blockDim.x) {
        const int cc = k % CW, j = k / CW;
        Cplx<T> z = a[cc * L + fpad(j)];
        z.re = z.re / n; z.im = z.im / n;
        A[(size_t)j * nx + c0 + cc] = z;
    }
}

// pass 3: inverse FFT along x, real part -> phi (pitched).
template <class T>
__global__ void __launch_bounds__(FFT_NT) fft_rows_inv_kernel(const Cplx<T>* __restrict__ A, int nx, int logn, const Cplx<T>* __restrict__ tw,
                                    T* __restrict__ phi, int pitch, const int* __restrict__ active) {
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Cplx<T>* a = reinterpret_cast<Cplx<T>*>(smem_raw);
    const int j = blockIdx.x;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) a[fpad(bitrev(i, logn))] = A[(size_t)j * nx + i];
    __syncthreads();
    fft_passes(a, nx, 1, tw);
    const T n = (T)nx;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) phi[(size_t)j * pitch + i] = a[fpad(i)].re / n;
}

// ---------------------------------------------------------------------------
// Red-black SOR, FP64 throughout.
// ---------------------------------------------------------------------------
struct SorArgs {
    int nx, ny;
    AxisMap ax, ay;
    double idx2, idy2, denom, omega, tol;
    int max_iter;
    const double* rhs;      // nx*ny contiguous
    double* phi;            // nx*ny contiguous
    double* part;           // gridDim.x partials
    double* part2;          // gridDim.x partials (residual)
    GridBarrier bar;
    int* iters_out;
    double* res_out;
    const int* active;
};

// Lexicographic SOR, the reference's own solve (compute_poisson_gravity_periodic,
// M2:178-237 and EH:288-386) in its own order, for parity runs.  One
// CTA.  A sweep runs as anti-diagonal wavefronts: the cells with i + j = d
// update together, d = 0 .. nx + ny - 2, with a barrier between diagonals.
// Of a cell's neighbours, west and south lie on diagonal d - 1 (already
// updated in this sweep), east and north on d + 1 (not yet), and a periodic
// wrap neighbour on d +- (n - 1): (0, j) reads (nx - 1, j) before this sweep
// updates it and (nx - 1, j) reads (0, j) after, as the row-major loop does;
// a clamped neighbour that is the cell itself is read before its update.  So
// every cell sees exactly the values the reference's loop sees.  The density
// mean and each sweep's mean of phi are summed by one thread in the
// reference's row-major order, and the update is the reference's expression,
// so phi is the reference's to the last bit.  Slow by design (nx + ny - 1
// barriers and an N-term sequential sum per sweep); the red-black kernel is
// the production solve.  tol > 0: stop after the first sweep whose max
// |lap(phi) - rhs|, taken inside the sweep from each cell's update as
// EH:335-368 does, is below tol.
struct SorLexArgs {
    int nx, ny, pitch;
    AxisMap ax, ay;
    double idx2, idy2, denom, omega, fourpiG, tol;
    double floor_rho;       // >= 0: density floored at it first (EH:307-313); < 0: as read (M2)
    int max_iter;
    double* rhs;            // nx*ny contiguous (written)
    double* phi;            // nx*ny contiguous (written)
    int* iters_out;
    double* res_out;
    const int* active;
};

template <class T, int NT>
__global__ void __launch_bounds__(NT) sor_lex_kernel(SorLexArgs a, const T* __restrict__ rho) {
    if (a.active && *a.active == 0) return;
    __shared__ double sh[NT / 32];
    __shared__ double s_val;
    const int nx = a.nx, ny = a.ny, N = nx * ny, tid = threadIdx.x;
    double* __restrict__ phi = a.phi;
    // rhobar and rhs = 4 pi G (rho - rhobar) (M2:187-194; EH:307-321 with the floor)
    auto dens = [&](int i, int j) {
        const double r = (double)rho[(size_t)j * a.pitch + i];
        return (a.floor_rho >= 0.0 && r < a.floor_rho) ? a.floor_rho : r;   // std::max(rho, floor_rho)
    };
    if (tid == 0) {
        double s = 0.0;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) s += dens(i, j);
        s_val = s / (double)N;
    }
    __syncthreads();
    const double rhobar = s_val;
    for (int j = 0; j < ny; j++)
        for (int i = tid; i < nx; i += NT) {
            const size_t q = (size_t)j * nx + i;
            a.rhs[q] = a.fourpiG * (dens(i, j) - rhobar);
            phi[q] = 0.0;
        }
    __syncthreads();
    int it = 0;
    double res = 0.0;
    for (; it < a.max_iter; ++it) {
        double r = 0.0;   // tol > 0: the residual taken inside the sweep (EH:335-368)
        for (int d = 0; d <= nx + ny - 2; ++d) {
            const int i0 = d - (ny - 1) > 0 ? d - (ny - 1) : 0, i1 = d < nx - 1 ? d : nx - 1;
            for (int i = i0 + tid; i <= i1; i += NT) {
                const int j = d - i;
                const size_t k = (size_t)j * nx + i;
                const double phiE = phi[(size_t)j * nx + a.ax.cell(i + 1)];
                const double phiW = phi[(size_t)j * nx + a.ax.cell(i - 1)];
                const double phiN = phi[(size_t)a.ay.cell(j + 1) * nx + i];
                const double phiS = phi[(size_t)a.ay.cell(j - 1) * nx + i];
                const double phi_new = ((phiE + phiW) * a.idx2 + (phiN + phiS) * a.idy2 - a.rhs[k]) / a.denom;
                const double v = phi[k] + a.omega * (phi_new - phi[k]);
                phi[k] = v;
                if (a.tol > 0.0) {
                    const double lap = (phiE - 2.0 * v + phiW) * a.idx2 + (phiN - 2.0 * v + phiS) * a.idy2;
                    r = fmax(r, fabs(lap - a.rhs[k]));
                }
            }
            __syncthreads();
        }
        // phibar in row-major order (M2:219-222)
        if (tid == 0) {
            double s = 0.0;
            for (int q = 0; q < N; q++) s += phi[q];
            s_val = s / (double)N;
        }
        __syncthreads();
        const double phibar = s_val;
        for (int q = tid; q < N; q += NT) phi[q] -= phibar;
        __syncthreads();
        if (a.tol > 0.0) {
            const double r0 = block_max<NT>(r, sh);   // valid in thread 0
            if (tid == 0) s_val = r0;
            __syncthreads();
            res = s_val;
            __syncthreads();   // s_val is rewritten by the next sweep's mean
            if (res < a.tol) { ++it; break; }
        }
    }
    if (tid == 0) {
        if (a.iters_out) *a.iters_out = it;
        if (a.res_out) *a.res_out = res;
    }
}

// max |lap(phi) - rhs| over the block's cells of the field phi - shift (the
// stored field with a pending mean removal applied on the fly)
template <int NT>
__device__ __forceinline__ double sor_residual_block(const SorArgs& a, double shift, double* sh) {
    double r = 0.0;
    const int N = a.nx * a.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < N; k += gridDim.x * NT) {
        const int i = k % a.nx, j = k / a.nx;
        const double c = a.phi[k] - shift;
        const double pE = a.phi[(size_t)j * a.nx + a.ax.cell(i + 1)] - shift;
        const double pW = a.phi[(size_t)j * a.nx + a.ax.cell(i - 1)] - shift;
        const double pN = a.phi[(size_t)a.ay.cell(j + 1) * a.nx + i] - shift;
        const double pS = a.phi[(size_t)a.ay.cell(j - 1) * a.nx + i] - shift;
        const double lap = (pE - 2.0 * c + pW) * a.idx2 + (pN - 2.0 * c + pS) * a.idy2;
        r = fmax(r, fabs(lap - a.rhs[k]));
    }
    return block_max<NT>(r, sh);
}

// One sweep = red update, black update, mean removal, and (tol > 0) the
// residual test.  The mean removal phi -= mean is not a pass of its own: the
// mean of a sweep stays pending (`m`) and every read of a value that the
// sweep has not rewritten subtracts it, which gives the same doubles as
// subtracting first (x - m is the value the reference stores), and x - 0.0 == x
// for the values already rewritten.  The density-independent part of the
// mean (the block partial sums) is formed in the black phase, which also reads
// the red cell of each of its indices, so a sweep needs two grid barriers
// (red, black) plus one for the residual when tol > 0.  A final pass applies
// the last pending mean.
template <int NT>
__global__ void __launch_bounds__(NT) sor_rb_kernel(SorArgs a) {
    if (a.active && *a.active == 0) return;
    __shared__ double sh[NT / 32];
    __shared__ double s_val;
    const unsigned nb = gridDim.x;
    const int N = a.nx * a.ny;
    const int half = (a.nx + 1) / 2;        // cells of one colour per row (upper bound)
    const int M = half * a.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < N; k += nb * NT) a.phi[k] = 0.0;
    if (!grid_sync(a.bar, nb)) return;
    // the mean of the block partial sums in block order (the same double in every block)
    auto block_mean = [&]() {
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (unsigned b = 0; b < nb; b++) t += a.part[b];
            s_val = t / (double)N;
        }
        __syncthreads();
        return s_val;
    };
    double m = 0.0;   // mean removal pending on every cell not yet rewritten in this sweep
    int it = 0;
    double res = 0.0;
    for (; it < a.max_iter; ++it) {
        // red: every value read is pending
        for (int k = blockIdx.x * NT + threadIdx.x; k < M; k += nb * NT) {
            const int j = k / half;
            const int i = 2 * (k % half) + (j & 1);
            if (i >= a.nx) continue;
            const size_t q = (size_t)j * a.nx + i;
            const double pE = a.phi[(size_t)j * a.nx + a.ax.cell(i + 1)] - m;
            const double pW = a.phi[(size_t)j * a.nx + a.ax.cell(i - 1)] - m;
            const double pN = a.phi[(size_t)a.ay.cell(j + 1) * a.nx + i] - m;
            const double pS = a.phi[(size_t)a.ay.cell(j - 1) * a.nx + i] - m;
            const double own = a.phi[q] - m;
            const double pn = ((pE + pW) * a.idx2 + (pN + pS) * a.idy2 - a.rhs[q]) / a.denom;
            a.phi[q] = own + a.omega * (pn - own);
        }
        if (!grid_sync(a.bar, nb)) return;
        // black: the red neighbours are rewritten; a clamped neighbour that is
        // the cell itself is still pending.  Sum every cell of the new field.
        double s = 0.0;
        for (int k = blockIdx.x * NT + threadIdx.x; k < M; k += nb * NT) {
            const int j = k / half;
            const int ir = 2 * (k % half) + (j & 1), i = 2 * (k % half) + ((j + 1) & 1);
            if (ir < a.nx) s += a.phi[(size_t)j * a.nx + ir];
            if (i >= a.nx) continue;
            const size_t q = (size_t)j * a.nx + i;
            const int iE = a.ax.cell(i + 1), iW = a.ax.cell(i - 1), jN = a.ay.cell(j + 1), jS = a.ay.cell(j - 1);
            const double pE = a.phi[(size_t)j * a.nx + iE] - (iE == i ? m : 0.0);
            const double pW = a.phi[(size_t)j * a.nx + iW] - (iW == i ? m : 0.0);
            const double pN = a.phi[(size_t)jN * a.nx + i] - (jN == j ? m : 0.0);
            const double pS = a.phi[(size_t)jS * a.nx + i] - (jS == j ? m : 0.0);
            const double own = a.phi[q] - m;
            const double pn = ((pE + pW) * a.idx2 + (pN + pS) * a.idy2 - a.rhs[q]) / a.denom;
            const double v = own + a.omega * (pn - own);
            a.phi[q] = v;
            s += v;
        }
        s = block_sum<NT>(s, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x] = s;
        if (!grid_sync(a.bar, nb)) return;
        m = block_mean();   // this sweep's mean, pending from here on
        if (a.tol > 0.0) {
            const double r = sor_residual_block<NT>(a, m, sh);
            if (threadIdx.x == 0) a.part2[blockIdx.x] = r;
            if (!grid_sync(a.bar, nb)) return;
            if (threadIdx.x == 0) {
                double mx = 0.0;
                for (unsigned b = 0; b < nb; b++) mx = fmax(mx, a.part2[b]);
                s_val = mx;
            }
            __syncthreads();
            res = s_val;
            __syncthreads();   // s_val is rewritten by the next block_mean
            // part and part2 are next written after at least one more grid
            // barrier, when every block has read them
            if (res < a.tol) { ++it; break; }
        }
    }
    // apply the last pending mean
    for (int k = blockIdx.x * NT + threadIdx.x; k < N; k += nb * NT) a.phi[k] -= m;
    if (!(a.tol > 0.0)) {
        if (!grid_sync(a.bar, nb)) return;
        const double r = sor_residual_block<NT>(a, 0.0, sh);
        if (threadIdx.x == 0) a.part2[blockIdx.x] = r;
        if (!grid_sync(a.bar, nb)) return;
        if (threadIdx.x == 0) {
            double mx = 0.0;
            for (unsigned b = 0; b < nb; b++) mx = fmax(mx, a.part2[b]);
            res = mx;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) { *a.iters_out = it; *a.res_out = res; }
}

// rhs = 4 pi G (rho - mean) (M2:187-194), mean from the density partial sums.
// floor_rho >= 0: the density is floored first (EH:312), and the partial sums
// must then be sums of the floored density.
template <class T>
__global__ void sor_rhs_kernel(const T* __restrict__ rho, int nx, int ny, int pitch, const double* __restrict__ rho_part,
                               int nparts, double fourpiG, double floor_rho, double* __restrict__ rhs,
                               const int* __restrict__ active) {
    if (active && *active == 0) return;
    __shared__ double s_mean;
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nparts; b++) s += rho_part[b];
        s_mean = s / ((double)nx * (double)ny);
    }
    __syncthreads();
    const double mean = s_mean;
    const int N = nx * ny;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        const int i = k % nx, j = k / nx;
        double r = (double)rho[(size_t)j * pitch + i];
        if (floor_rho >= 0.0) r = vmax(r, floor_rho);
        rhs[k] = fourpiG * (r - mean);
    }
}

// copy the contiguous FP64 phi into the pitched T field the stage kernel reads
template <class T>
__global__ void phi_to_field_kernel(const double* __restrict__ phi, int nx, int ny, T* __restrict__ out, int pitch,
                                    const int* __restrict__ active) {
    if (active && *active == 0) return;
    const int N = nx * ny;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        const int i = k % nx, j = k / nx;
        out[(size_t)j * pitch + i] = (T)phi[k];
    }
}

// g = -grad(phi) (M2:225-235), written pitched, for the host-facing gravity call
template <class T>
__global__ void gravity_from_phi_kernel(const T* __restrict__ phi, int nx, int ny, int pitch, AxisMap ax, AxisMap ay,
                                        T two_dx, T two_dy, T* __restrict__ gx, T* __restrict__ gy) {
    const int N = nx * ny;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) {
        const int i = k % nx, j = k / nx;
        const size_t q = (size_t)j * pitch + i;
        gx[q] = -(phi[(size_t)j * pitch + ax.cell(i + 1)] - phi[(size_t)j * pitch + ax.cell(i - 1)]) / two_dx;
        gy[q] = -(phi[(size_t)ay.cell(j + 1) * pitch + i] - phi[(size_t)ay.cell(j - 1) * pitch + i]) / two_dy;
    }
}

}  // namespace ccb
