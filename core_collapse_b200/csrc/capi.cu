// C ABI of libcc_b200 (declared in include/cc_step.h): handle lifetime, state
// transfer, and the 2D MHD step orchestration on one CUDA stream.
//
// Per step the device runs (mhd2d_resistive_hlld_ct_gravity.cpp:1111-1117, 838-869):
//   Poisson(U^n.rho) -> phi;  dt = finalize(CFL partials) (clamped to t_end);
//   stage 1: U^n -> S1 (pre-Joule);  Poisson(S1.rho) -> phi;
//   stage 2: Joule(S1) -> S2 (pre-Joule);
//   average: U^{n+1} = floors(0.5 (U^n + Joule(S2))), which also emits the CFL
//            and density partials of U^{n+1} for the next step;  t += dt.
// Three pitched state buffers rotate (U^n, S1, S2); dt, t and the "active"
// flag (t < t_end) live on the device, so a run of steps needs no host sync
// and is captured as a CUDA graph (three steps = one buffer rotation).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/cc_step.h"
#include "checkpoint.h"
#include "fft_tables.h"
#include "mhd2d_launch.h"
#include "handle.h"

using namespace ccb;

namespace {

bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Rows per segment of the column-march stage kernel: as long as possible (each
// segment pays a half step to build its carried rows), but short enough that
// the strips x segments fill 148 SMs x 4 resident CTAs about twice; a
// multiple of the 8-row march step, 16 to 128 rows.
int default_march_rows(int nx, int ny) {
    const long strips = (nx + 31) / 32;
    long rows = (long)ny * strips / (148L * 4 * 2);
    rows = rows / 8 * 8;
    if (rows < 16) rows = 16;
    if (rows > 128) rows = 128;
    return (int)rows;
}
int ilog2(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }

// --------------------------------------------------------------------------
// 2D MHD solver state, one instantiation per precision
// --------------------------------------------------------------------------
struct Mhd2dBase {
    virtual ~Mhd2dBase() {}
    virtual int init() = 0;
    virtual int upload(const double* const* f) = 0;
    virtual int download(double* const* f) = 0;
    virtual int gravity(double* gx, double* gy) = 0;
    virtual int compute_dt(double* dt) = 0;
    virtual int rk2_step(const double* gx, const double* gy, double dt) = 0;
    virtual int advance(int nsteps, double* t) = 0;
    virtual int diagnostics(cc_diag* d) = 0;
    virtual int derived(double* const* out) = 0;
    virtual int get_clock(double* t, long long* steps) = 0;
    virtual int set_clock(double t, long long steps) = 0;
    virtual const cc_mhd2d_params& params() const = 0;
    virtual int set_stage_kernel(int kind, int seg_rows) = 0;
};

template <class T> struct Mhd2d : Mhd2dBase {
    cc_handle* h;
    cc_mhd2d_params p;
    M2Const<T> c;
    int P = 0;
    size_t plane = 0;
    void* block = nullptr;
    Fields<T> buf[3];
    // compensated FP32 state (p.compensated): the rounding residual of every plane of buf[b] in lbuf[b]
    bool comp = false;
    void* lblock = nullptr;
    Fields<T> lbuf[3];
    // stage kernel: CC_STAGE_TILE (the default; FP64's only form) or CC_STAGE_MARCH (FP32)
    int stage_kind = CC_STAGE_TILE;
    int march_rows = 0;   // 0: from the grid (init)
    int cur = 0;
    T* phi = nullptr;
    T* gxa = nullptr;
    T* gya = nullptr;
    Cplx<T>* fftA = nullptr;
    // FP64: twiddles x fwd, x inv, y fwd, y inv; FP32: roots of nx in tw[0], of ny in tw[2]
    Cplx<T>* tw[4] = {nullptr, nullptr, nullptr, nullptr};
    double* rhs = nullptr;
    double* sphi = nullptr;
    double* scal = nullptr;   // small device scalars
    double* spd_part = nullptr;
    double* rho_part = nullptr;
    double* diag_part = nullptr;
    double* sor_part = nullptr;
    double* sor_part2 = nullptr;
    double* staging = nullptr;
    unsigned int* bar = nullptr;  // count, gen
    int* iflags = nullptr;        // active, bar_err, sor_iters, fft_copy_err
    double* dt_dev = nullptr;
    double* t_dev = nullptr;
    double* sor_res = nullptr;
    long long* steps_dev = nullptr;
    double* derived_dev = nullptr;   // 10 planes of Nx*Ny, allocated at the first cc_mhd2d_derived
    bool loaded = false;
    bool rho_part_valid = false;   // rho_part / spd_part describe buf[cur]
    bool phi_valid = false;        // phi is the Poisson solution of buf[cur].rho
    cudaGraphExec_t graph3 = nullptr;
    cudaStream_t graph_stream = nullptr;
    int graph_cur = -1;

    explicit Mhd2d(cc_handle* hh, const cc_mhd2d_params& pp) : h(hh), p(pp) {}
    cc_handle* this_handle() { return h; }
    cudaStream_t st() const { return h->stream; }
    int* active() { return iflags; }

    ~Mhd2d() override {
        if (graph3) cudaGraphExecDestroy(graph3);
        void* ptrs[] = {block, lblock, phi, gxa, gya, fftA, tw[0], tw[1], tw[2], tw[3], rhs, sphi, scal, spd_part, rho_part,
                        diag_part, sor_part, sor_part2, staging, bar, iflags, steps_dev, derived_dev};
        for (void* q : ptrs)
            if (q) cudaFree(q);
    }

    int init() override {
        const int nx = p.Nx, ny = p.Ny;
        const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
        c.gamma = (T)p.gamma;
        c.gm1 = (T)p.gamma - (T)1.0;
        c.floor_rho = (T)p.floor_rho;
        c.floor_P = (T)p.floor_P;
        c.eta = (T)p.eta;
        c.dx = (T)dx; c.dy = (T)dy;
        c.inv_dx = (T)(1.0 / dx); c.inv_dy = (T)(1.0 / dy);
        c.idx2 = (T)(1.0 / (dx * dx)); c.idy2 = (T)(1.0 / (dy * dy));
        c.two_dx = (T)(2.0 * dx); c.two_dy = (T)(2.0 * dy);
        c.nx = nx; c.ny = ny;
        P = ((nx + 1 + 31) / 32) * 32;
        c.pitch = P;
        c.ax = AxisMap{nx, p.periodic_x ? 1 : 0};
        c.ay = AxisMap{ny, p.periodic_y ? 1 : 0};
        c.gravity_on = p.gravity_on ? 1 : 0;
        c.resistive = (p.eta > 0.0) ? 1 : 0;
        plane = (size_t)P * (ny + 1);
        march_rows = default_march_rows(nx, ny);
        CC_CUDA(M2Launch<T>::prepare(nx, ny));

        if (p.compensated && sizeof(T) != 4)
            return fail(h, CC_ERR_UNSUPPORTED, "the compensated update is an option of the FP32 path");
        comp = p.compensated != 0;
        CC_CUDA(cudaMalloc(&block, sizeof(T) * plane * 24));
        CC_CUDA(cudaMemsetAsync(block, 0, sizeof(T) * plane * 24, st()));
        for (int b = 0; b < 3; b++) {
            T* base = reinterpret_cast<T*>(block) + (size_t)b * 8 * plane;
            buf[b] = Fields<T>{base, base + plane, base + 2 * plane, base + 3 * plane,
                               base + 4 * plane, base + 5 * plane, base + 6 * plane, base + 7 * plane};
        }
        if (comp) {
            CC_CUDA(cudaMalloc(&lblock, sizeof(T) * plane * 24));
            CC_CUDA(cudaMemsetAsync(lblock, 0, sizeof(T) * plane * 24, st()));
            for (int b = 0; b < 3; b++) {
                T* base = reinterpret_cast<T*>(lblock) + (size_t)b * 8 * plane;
                lbuf[b] = Fields<T>{base, base + plane, base + 2 * plane, base + 3 * plane,
                                    base + 4 * plane, base + 5 * plane, base + 6 * plane, base + 7 * plane};
            }
        }
        CC_CUDA(cudaMalloc(&phi, sizeof(T) * plane));
        CC_CUDA(cudaMemsetAsync(phi, 0, sizeof(T) * plane, st()));
        CC_CUDA(cudaMalloc(&spd_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&rho_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&diag_part, sizeof(double) * RED_BLOCKS * 7));
        CC_CUDA(cudaMalloc(&staging, sizeof(double) * (size_t)(nx + 1) * (ny + 1)));
        CC_CUDA(cudaMalloc(&scal, sizeof(double) * 8));
        CC_CUDA(cudaMemsetAsync(scal, 0, sizeof(double) * 8, st()));
        dt_dev = scal; t_dev = scal + 1; sor_res = scal + 2;
        CC_CUDA(cudaMalloc(&steps_dev, sizeof(long long)));
        CC_CUDA(cudaMemsetAsync(steps_dev, 0, sizeof(long long), st()));
        CC_CUDA(cudaMalloc(&iflags, sizeof(int) * 4));
        int init_flags[4] = {1, 0, 0, 0};
        CC_CUDA(cudaMemcpyAsync(iflags, init_flags, sizeof(init_flags), cudaMemcpyHostToDevice, st()));

        if (p.gravity_on) {
            if (p.poisson_kind == CC_POISSON_FFT) {
                if (!p.periodic_x || !p.periodic_y)
                    return fail(h, CC_ERR_UNSUPPORTED, "FFT Poisson needs periodic_x and periodic_y");
                // power of two >= 4: the column pass works on strips of 2 (FP64) or 4 (FP32) columns
                if (!is_pow2(nx) || !is_pow2(ny) || nx < 4 || ny < 4)
                    return fail(h, CC_ERR_UNSUPPORTED, "FFT Poisson needs power-of-two Nx, Ny >= 4");
                if ((size_t)nx * sizeof(Cplx<T>) > 200 * 1024 || (size_t)ny * sizeof(Cplx<T>) * (sizeof(T) == 8 ? 2 : 4) > 200 * 1024)
                    return fail(h, CC_ERR_UNSUPPORTED, "FFT line does not fit in shared memory");
                if (sizeof(T) == 4 && (nx > FFT32_MAXN || ny > FFT32_MAXN))
                    return fail(h, CC_ERR_UNSUPPORTED, "FP32 FFT Poisson supports Nx, Ny <= 8192");
                if constexpr (sizeof(T) == 4) {
                    // FP32: half-spectrum work array (kx-major), root tables of nx and ny in tw[0], tw[2]
                    const size_t w = (size_t)fft32_half_lines(nx);
                    CC_CUDA(cudaMalloc(&fftA, sizeof(Cplx<T>) * w * ny));
                    const int ns[2] = {nx, ny};
                    for (int k = 0; k < 2; k++) {
                        const std::vector<float> t = fft32_roots(ns[k]);
                        CC_CUDA(cudaMalloc(&tw[2 * k], sizeof(float) * t.size()));
                        CC_CUDA(cudaMemcpyAsync(tw[2 * k], t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice, st()));
                    }
                } else {
                    CC_CUDA(cudaMalloc(&fftA, sizeof(Cplx<T>) * (size_t)nx * ny));
                    const int ns[4] = {nx, nx, ny, ny};
                    for (int k = 0; k < 4; k++) {
                        std::vector<double> t = twiddle_table(ns[k], k & 1);
                        std::vector<T> tt(t.begin(), t.end());
                        CC_CUDA(cudaMalloc(&tw[k], sizeof(T) * tt.size()));
                        CC_CUDA(cudaMemcpyAsync(tw[k], tt.data(), sizeof(T) * tt.size(), cudaMemcpyHostToDevice, st()));
                    }
                }
            } else if (p.poisson_kind == CC_POISSON_SOR_LEX) {
                CC_CUDA(cudaMalloc(&rhs, sizeof(double) * (size_t)nx * ny));
                CC_CUDA(cudaMalloc(&sphi, sizeof(double) * (size_t)nx * ny));
            } else if (p.poisson_kind == CC_POISSON_SOR) {
                if ((p.periodic_x && (nx & 1)) || (p.periodic_y && (ny & 1)))
                    return fail(h, CC_ERR_UNSUPPORTED, "red-black SOR needs an even extent along periodic axes");
                CC_CUDA(cudaMalloc(&rhs, sizeof(double) * (size_t)nx * ny));
                CC_CUDA(cudaMalloc(&sphi, sizeof(double) * (size_t)nx * ny));
                CC_CUDA(cudaMalloc(&sor_part, sizeof(double) * 4096));
                CC_CUDA(cudaMalloc(&sor_part2, sizeof(double) * 4096));
                CC_CUDA(cudaMalloc(&bar, sizeof(unsigned int) * 2));
                CC_CUDA(cudaMemsetAsync(bar, 0, sizeof(unsigned int) * 2, st()));
            } else {
                return fail(h, CC_ERR_ARG, "unknown poisson_kind");
            }
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    void invalidate_graph() {
        if (graph3) { cudaGraphExecDestroy(graph3); graph3 = nullptr; }
    }

    int upload(const double* const* f) override {
        const int nx = p.Nx, ny = p.Ny;
        const int w[8] = {nx, nx, nx, nx, nx, nx, nx + 1, nx};
        const int hh[8] = {ny, ny, ny, ny, ny, ny, ny, ny + 1};
        T* dst[8] = {buf[cur].rho, buf[cur].mx, buf[cur].my, buf[cur].mz, buf[cur].E, buf[cur].Bz, buf[cur].bx, buf[cur].by};
        T* ldst[8] = {lbuf[cur].rho, lbuf[cur].mx, lbuf[cur].my, lbuf[cur].mz, lbuf[cur].E, lbuf[cur].Bz, lbuf[cur].bx, lbuf[cur].by};
        for (int k = 0; k < 8; k++) {
            if (!f[k]) return fail(h, CC_ERR_ARG, "null state array");
            CC_CUDA(cudaMemcpyAsync(staging, f[k], sizeof(double) * (size_t)w[k] * hh[k], cudaMemcpyHostToDevice, st()));
            if (comp)
                CC_CUDA(M2Launch<T>::pack_in_split(staging, dst[k], ldst[k], w[k], hh[k], P, st()));
            else
                CC_CUDA(M2Launch<T>::pack_in(staging, dst[k], w[k], hh[k], P, st()));
        }
        loaded = true;
        rho_part_valid = false;
        phi_valid = false;
        return CC_OK;
    }

    int download(double* const* f) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        const int nx = p.Nx, ny = p.Ny;
        const int w[8] = {nx, nx, nx, nx, nx, nx, nx + 1, nx};
        const int hh[8] = {ny, ny, ny, ny, ny, ny, ny, ny + 1};
        const T* src[8] = {buf[cur].rho, buf[cur].mx, buf[cur].my, buf[cur].mz, buf[cur].E, buf[cur].Bz, buf[cur].bx, buf[cur].by};
        const T* lsrc[8] = {lbuf[cur].rho, lbuf[cur].mx, lbuf[cur].my, lbuf[cur].mz, lbuf[cur].E, lbuf[cur].Bz, lbuf[cur].bx, lbuf[cur].by};
        for (int k = 0; k < 8; k++) {
            if (!f[k]) continue;
            if (comp)
                CC_CUDA(M2Launch<T>::pack_out_sum(src[k], lsrc[k], staging, w[k], hh[k], P, st()));
            else
                CC_CUDA(M2Launch<T>::pack_out(src[k], staging, w[k], hh[k], P, st()));
            CC_CUDA(cudaMemcpyAsync(f[k], staging, sizeof(double) * (size_t)w[k] * hh[k], cudaMemcpyDeviceToHost, st()));
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return check_flags();
    }

    int check_flags() {
        int fl[4];
        CC_CUDA(cudaMemcpy(fl, iflags, sizeof(fl), cudaMemcpyDeviceToHost));
        if (fl[1]) return fail(h, CC_ERR_CUDA, "SOR grid barrier timed out");
        if (fl[3]) return fail(h, CC_ERR_CUDA, "FFT column pass: a bulk-copy wait timed out");
        return CC_OK;
    }

    // density sum + CFL partials of buf[cur]
    int ensure_partials() {
        if (rho_part_valid) return CC_OK;
        CC_CUDA(M2Launch<T>::speeds(c, buf[cur], spd_part, rho_part, st()));
        count(1);
        rho_part_valid = true;
        return CC_OK;
    }

    // Poisson on a density field; rho_part must hold its sum.  Writes phi.
    int solve(const T* rho) {
        if (!p.gravity_on) return CC_OK;
        h->perf.poisson_solves += 1;
        const int nx = p.Nx, ny = p.Ny;
        if (p.poisson_kind == CC_POISSON_FFT) {
            if constexpr (sizeof(T) == 4)
                CC_CUDA(M2Launch<T>::fft32_solve(rho, P, rho_part, nx, ny, reinterpret_cast<const float2*>(tw[0]),
                                                 reinterpret_cast<const float2*>(tw[2]), p.x1 - p.x0, p.y1 - p.y0,
                                                 p.G, reinterpret_cast<float2*>(fftA), phi, active(), st(),
                                                 iflags + 3));
            else
                CC_CUDA(M2Launch<T>::fft_solve(rho, P, rho_part, nx, ny, ilog2(nx), ilog2(ny), tw[0], tw[1], tw[2],
                                               tw[3], p.x1 - p.x0, p.y1 - p.y0, p.G, fftA, phi, active(), st()));
            count(3);
        } else if (p.poisson_kind == CC_POISSON_SOR_LEX) {
            const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
            SorLexArgs a;
            a.nx = nx; a.ny = ny; a.pitch = P; a.ax = c.ax; a.ay = c.ay;
            a.idx2 = 1.0 / (dx * dx); a.idy2 = 1.0 / (dy * dy);
            a.denom = 2.0 * (a.idx2 + a.idy2);
            a.omega = p.sor_omega; a.fourpiG = 4.0 * M_PI * p.G; a.tol = p.sor_tol; a.max_iter = p.sor_iters;
            a.floor_rho = -1.0;   // M2 solves with the stored density (M2:187-194)
            a.rhs = rhs; a.phi = sphi; a.iters_out = iflags + 2; a.res_out = sor_res; a.active = active();
            CC_CUDA(launch_sor_lex<T>(a, rho, st()));
            CC_CUDA(M2Launch<T>::phi_to_field(sphi, nx, ny, phi, P, active(), st()));
            count(2);
        } else {
            CC_CUDA(M2Launch<T>::sor_rhs(rho, nx, ny, P, rho_part, 4.0 * M_PI * p.G, -1.0, rhs, active(), st()));
            const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
            SorArgs a;
            a.nx = nx; a.ny = ny; a.ax = c.ax; a.ay = c.ay;
            a.idx2 = 1.0 / (dx * dx); a.idy2 = 1.0 / (dy * dy);
            a.denom = 2.0 * (a.idx2 + a.idy2);
            a.omega = p.sor_omega; a.tol = p.sor_tol; a.max_iter = p.sor_iters;
            a.rhs = rhs; a.phi = sphi; a.part = sor_part; a.part2 = sor_part2;
            a.bar = GridBarrier{bar, bar + 1, iflags + 1};
            a.iters_out = iflags + 2; a.res_out = sor_res; a.active = active();
            int nb = 0;
            CC_CUDA(launch_sor(a, &nb, st()));
            CC_CUDA(M2Launch<T>::phi_to_field(sphi, nx, ny, phi, P, active(), st()));
            count(3);
        }
        return CC_OK;
    }

    int gravity(double* gx, double* gy) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        const int nx = p.Nx, ny = p.Ny;
        if (p.gravity_on) {
            int r = ensure_partials();
            if (r) return r;
            CC_CUDA(launch_set_scalar(dt_dev, 0.0, st()));
            int one = 1;
            CC_CUDA(cudaMemcpyAsync(iflags, &one, sizeof(int), cudaMemcpyHostToDevice, st()));
            r = solve(buf[cur].rho);
            if (r) return r;
            phi_valid = true;
        }
        if (gx || gy) {
            if (!gxa) {
                CC_CUDA(cudaMalloc(&gxa, sizeof(T) * plane));
                CC_CUDA(cudaMalloc(&gya, sizeof(T) * plane));
            }
            if (p.gravity_on) {
                CC_CUDA(M2Launch<T>::gravity_from_phi(phi, nx, ny, P, c.ax, c.ay, c.two_dx, c.two_dy, gxa, gya, st()));
            } else {
                CC_CUDA(cudaMemsetAsync(gxa, 0, sizeof(T) * plane, st()));
                CC_CUDA(cudaMemsetAsync(gya, 0, sizeof(T) * plane, st()));
            }
            T* src[2] = {gxa, gya};
            double* dst[2] = {gx, gy};
            for (int k = 0; k < 2; k++) {
                if (!dst[k]) continue;
                CC_CUDA(M2Launch<T>::pack_out(src[k], staging, nx, ny, P, st()));
                CC_CUDA(cudaMemcpyAsync(dst[k], staging, sizeof(double) * (size_t)nx * ny, cudaMemcpyDeviceToHost, st()));
            }
            CC_CUDA(cudaStreamSynchronize(st()));
        }
        return check_flags();
    }

    DtSpec dtspec(bool clamp) const {
        const double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
        DtSpec d;
        d.cfl = p.cfl; d.hmin = vmin(dx, dy); d.eta = p.eta; d.t_end = p.t_end; d.clamp_to_end = clamp ? 1 : 0;
        d.seed = 1e-14; d.end_eps = 0.0; d.check = 0; d.cap = 1;
        return d;
    }

    int compute_dt(double* dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        int r = ensure_partials();
        if (r) return r;
        CC_CUDA(launch_dt_finalize(spd_part, dtspec(false), dt_dev, t_dev, active(), st()));
        CC_CUDA(cudaMemcpyAsync(dt, dt_dev, sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    void count(int n) { h->perf.kernel_launches += n; }

    // one stage-kernel launch from buf[bi] to buf[bo], bracketed by CUDA events when profiling
    int stage(int bi, int bo, bool defer, int gmode, const T* ga, const T* gb) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (h->profiling) {
            CC_CUDA(cudaEventCreate(&e0));
            CC_CUDA(cudaEventCreate(&e1));
            CC_CUDA(cudaEventRecord(e0, st()));
        }
        if (stage_kind == CC_STAGE_MARCH)
            CC_CUDA(M2Launch<T>::stage_march(c, buf[bi], buf[bo], comp ? &lbuf[bi] : nullptr,
                                             comp ? &lbuf[bo] : nullptr, defer, gmode, ga, gb, dt_dev, active(),
                                             march_rows, st()));
        else if (comp)
            CC_CUDA(M2Launch<T>::stage_comp(c, buf[bi], buf[bo], lbuf[bi], lbuf[bo], defer, gmode, ga, gb, dt_dev,
                                            active(), st()));
        else
            CC_CUDA(M2Launch<T>::stage(c, buf[bi], buf[bo], defer, gmode, ga, gb, dt_dev, active(), st()));
        count(1);
        if (h->profiling) {
            CC_CUDA(cudaEventRecord(e1, st()));
            h->timed.emplace_back(e0, e1);
        }
        return CC_OK;
    }

    // stage 1 (gravity per gmode1), Poisson on S1, stage 2, average; dt in dt_dev
    int step_body(int gmode1) {
        const int a = cur, b = (cur + 1) % 3, d = (cur + 2) % 3;
        const int g2 = p.gravity_on ? GRAV_PHI : GRAV_NONE;
        int r = stage(a, b, false, gmode1, gmode1 == GRAV_ARRAYS ? gxa : phi, gmode1 == GRAV_ARRAYS ? gya : nullptr);
        if (r) return r;
        if (p.gravity_on) {
            CC_CUDA(M2Launch<T>::rho_sum(c, buf[b].rho, rho_part, st()));
            count(1);
            r = solve(buf[b].rho);
            if (r) return r;
        }
        r = stage(b, d, true, g2, phi, nullptr);
        if (r) return r;
        if (comp)
            CC_CUDA(M2Launch<T>::average_comp(c, buf[a], buf[d], buf[b], lbuf[a], lbuf[d], lbuf[b], dt_dev, active(),
                                              spd_part, rho_part, st()));
        else
            CC_CUDA(M2Launch<T>::average(c, buf[a], buf[d], buf[b], dt_dev, active(), spd_part, rho_part, st()));
        count(1);
        h->perf.steps += 1;
        cur = b;
        rho_part_valid = true;
        phi_valid = false;
        return CC_OK;
    }

    int rk2_step(const double* gx, const double* gy, double dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        int gmode1 = GRAV_NONE;
        if (p.gravity_on) {
            if (gx && gy) {
                if (!gxa) {
                    CC_CUDA(cudaMalloc(&gxa, sizeof(T) * plane));
                    CC_CUDA(cudaMalloc(&gya, sizeof(T) * plane));
                }
                const double* src[2] = {gx, gy};
                T* dst[2] = {gxa, gya};
                for (int k = 0; k < 2; k++) {
                    CC_CUDA(cudaMemcpyAsync(staging, src[k], sizeof(double) * (size_t)p.Nx * p.Ny, cudaMemcpyHostToDevice, st()));
                    CC_CUDA(M2Launch<T>::pack_in(staging, dst[k], p.Nx, p.Ny, P, st()));
                }
                gmode1 = GRAV_ARRAYS;
            } else if (gx || gy) {
                return fail(h, CC_ERR_ARG, "pass both gx and gy, or neither");
            } else {
                if (!phi_valid) return fail(h, CC_ERR_STATE, "no device gravity for this state: call cc_mhd2d_compute_gravity first");
                gmode1 = GRAV_PHI;
            }
        }
        int one = 1;
        CC_CUDA(cudaMemcpyAsync(iflags, &one, sizeof(int), cudaMemcpyHostToDevice, st()));
        CC_CUDA(launch_set_scalar(dt_dev, dt, st()));
        invalidate_graph();
        int r = step_body(gmode1);
        if (r) return r;
        CC_CUDA(cudaStreamSynchronize(st()));
        return check_flags();
    }

    // one step of the main() loop on the device
    int device_step() {
        int r = ensure_partials();
        if (r) return r;
        if (p.gravity_on) {
            r = solve(buf[cur].rho);
            if (r) return r;
        }
        CC_CUDA(launch_dt_finalize(spd_part, dtspec(true), dt_dev, t_dev, active(), st()));
        count(1);
        r = step_body(p.gravity_on ? GRAV_PHI : GRAV_NONE);
        if (r) return r;
        CC_CUDA(launch_clock(t_dev, dt_dev, active(), steps_dev, st()));
        count(1);
        return CC_OK;
    }

    // SOR uses a cooperative launch and profiling records events per launch:
    // both run eagerly
    bool graph_ok() const { return !(p.gravity_on && p.poisson_kind == CC_POISSON_SOR) && !h->profiling; }
    cc_perf graph_delta{};   // counters added by one replay of graph3

    int advance(int nsteps, double* t) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        if (nsteps < 0) return fail(h, CC_ERR_ARG, "nsteps < 0");
        if (t) CC_CUDA(launch_set_scalar(t_dev, *t, st()));
        int r = ensure_partials();
        if (r) return r;
        int done = 0;
        if (graph_ok() && nsteps >= 3) {
            if (!graph3 || graph_cur != cur || graph_stream != st()) {
                invalidate_graph();
                const int start = cur;
                cudaGraph_t g = nullptr;
                const cc_perf before = h->perf;
                CC_CUDA(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
                int rr = CC_OK;
                for (int k = 0; k < 3 && rr == CC_OK; k++) rr = device_step();
                cudaError_t e = cudaStreamEndCapture(st(), &g);
                cur = start;
                graph_delta.kernel_launches = h->perf.kernel_launches - before.kernel_launches;
                graph_delta.poisson_solves = h->perf.poisson_solves - before.poisson_solves;
                graph_delta.steps = h->perf.steps - before.steps;
                h->perf = before;   // captured, not run: counted per replay below
                if (rr) { if (g) cudaGraphDestroy(g); return rr; }
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
                e = cudaGraphInstantiate(&graph3, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
                graph_cur = start;
                graph_stream = st();
            }
            while (nsteps - done >= 3) {
                CC_CUDA(cudaGraphLaunch(graph3, st()));
                h->perf.kernel_launches += graph_delta.kernel_launches;
                h->perf.poisson_solves += graph_delta.poisson_solves;
                h->perf.steps += graph_delta.steps;
                done += 3;
            }
            rho_part_valid = true;
            phi_valid = false;
        }
        for (; done < nsteps; ++done) {
            r = device_step();
            if (r) return r;
        }
        if (t) {
            CC_CUDA(cudaMemcpyAsync(t, t_dev, sizeof(double), cudaMemcpyDeviceToHost, st()));
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return check_flags();
    }

    const cc_mhd2d_params& params() const override { return p; }

    int set_stage_kernel(int kind, int seg_rows) override {
        if (kind != CC_STAGE_TILE && kind != CC_STAGE_MARCH) return fail(h, CC_ERR_ARG, "unknown stage kernel");
        if (kind == CC_STAGE_MARCH && sizeof(T) != 4)
            return fail(h, CC_ERR_UNSUPPORTED, "the column-march stage kernel is an FP32 kernel");
        if (seg_rows < 0) return fail(h, CC_ERR_ARG, "seg_rows < 0");
        stage_kind = kind;
        march_rows = seg_rows > 0 ? seg_rows : default_march_rows(p.Nx, p.Ny);
        invalidate_graph();
        return CC_OK;
    }

    int derived(double* const* out) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        const size_t n = (size_t)p.Nx * p.Ny;
        if (!derived_dev) CC_CUDA(cudaMalloc(&derived_dev, sizeof(double) * n * 10));
        CC_CUDA(M2Launch<T>::derived(c, buf[cur], derived_dev, st()));
        for (int k = 0; k < 10; k++)
            if (out[k])
                CC_CUDA(cudaMemcpyAsync(out[k], derived_dev + k * n, sizeof(double) * n, cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return check_flags();
    }

    int get_clock(double* t, long long* steps) override {
        CC_CUDA(cudaMemcpyAsync(t, t_dev, sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaMemcpyAsync(steps, steps_dev, sizeof(long long), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int set_clock(double t, long long steps) override {
        CC_CUDA(launch_set_scalar(t_dev, t, st()));
        CC_CUDA(cudaMemcpyAsync(steps_dev, &steps, sizeof(long long), cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int diagnostics(cc_diag* d) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        CC_CUDA(M2Launch<T>::diag(c, buf[cur], diag_part, st()));
        std::vector<double> part(RED_BLOCKS * 7);
        CC_CUDA(cudaMemcpyAsync(part.data(), diag_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st()));
        double sc[8];
        CC_CUDA(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st()));
        long long steps = 0;
        CC_CUDA(cudaMemcpyAsync(&steps, steps_dev, sizeof(steps), cudaMemcpyDeviceToHost, st()));
        int fl[4];
        CC_CUDA(cudaMemcpyAsync(fl, iflags, sizeof(fl), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        double s[5] = {0, 0, 0, 0, 0}, dmax = 0.0, nonf = 0.0;
        for (int m = 0; m < 5; m++)
            for (int b = 0; b < RED_BLOCKS; b++) s[m] += part[m * RED_BLOCKS + b];
        for (int b = 0; b < RED_BLOCKS; b++) {
            dmax = std::fmax(dmax, part[5 * RED_BLOCKS + b]);
            nonf = std::fmax(nonf, part[6 * RED_BLOCKS + b]);
        }
        const double dV = ((p.x1 - p.x0) / p.Nx) * ((p.y1 - p.y0) / p.Ny);
        std::memset(d, 0, sizeof(*d));
        d->mass = s[0] * dV; d->mom_x = s[1] * dV; d->mom_y = s[2] * dV; d->mom_z = s[3] * dV; d->energy = s[4] * dV;
        d->max_divB = dmax;
        d->t = sc[1];
        d->dt_last = sc[0];
        d->steps = steps;
        d->poisson_iters = fl[2];
        d->poisson_residual = sc[2];
        d->nonfinite = nonf > 0.0 ? 1 : 0;
        if (fl[1]) return fail(h, CC_ERR_CUDA, "SOR grid barrier timed out");
        if (fl[3]) return fail(h, CC_ERR_CUDA, "FFT column pass: a bulk-copy wait timed out");
        return CC_OK;
    }
};

struct Mhd2dHandle : cc_handle {
    std::unique_ptr<Mhd2dBase> impl;
};

// checkpoint file helpers
constexpr char CK_MAGIC[9] = "CCB2DCK1";
constexpr uint32_t CK_VERSION = 1;

std::vector<size_t> ck_sizes(const cc_mhd2d_params& p) {
    const size_t nx = (size_t)p.Nx, ny = (size_t)p.Ny, n = nx * ny;
    return {n, n, n, n, n, n, (nx + 1) * ny, nx * (ny + 1)};
}

Mhd2dBase* m2(cc_handle* h) {
    if (!h || h->kind != KIND_MHD2D) return nullptr;
    return static_cast<Mhd2dHandle*>(h)->impl.get();
}

}  // namespace

extern "C" {

void cc_mhd2d_params_default(cc_mhd2d_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma = 5.0 / 3.0; p->cfl = 0.45;
    p->x0 = 0.0; p->x1 = 1.0; p->y0 = 0.0; p->y1 = 1.0;
    p->Nx = 192; p->Ny = 192;
    p->t_end = 0.35; p->dt_store = 1e-3;
    p->floor_rho = 1e-10; p->floor_P = 1e-10;
    p->periodic_x = 1; p->periodic_y = 1;
    p->eta = 5e-4;
    p->gravity_on = 1; p->G = 8.0; p->softening = 1e-4;
    p->sor_iters = 600; p->sor_omega = 1.8;
    p->sor_tol = 0.0; p->poisson_kind = CC_POISSON_SOR; p->precision = CC_FP64;
}

int cc_mhd2d_create(const cc_mhd2d_params* p, cc_handle** out) {
    if (!p || !out) return CC_ERR_ARG;
    *out = nullptr;
    if (p->Nx < 2 || p->Ny < 2) return CC_ERR_ARG;
    if (!(p->x1 > p->x0) || !(p->y1 > p->y0)) return CC_ERR_ARG;
    if (p->precision != CC_FP64 && p->precision != CC_FP32) return CC_ERR_ARG;
    auto h = std::make_unique<Mhd2dHandle>();
    h->kind = KIND_MHD2D;
    if (cudaGetDevice(&h->device) != cudaSuccess) return CC_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return CC_ERR_CUDA;
    h->stream = h->own;
    if (p->precision == CC_FP64) h->impl = std::make_unique<Mhd2d<double>>(h.get(), *p);
    else h->impl = std::make_unique<Mhd2d<float>>(h.get(), *p);
    int r = h->impl->init();
    if (r != CC_OK) {
        // keep the handle so the caller can read the message, then the caller destroys it
        *out = h.release();
        return r;
    }
    *out = h.release();
    return CC_OK;
}

int cc_destroy(cc_handle* h) {
    if (!h) return CC_ERR_ARG;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    delete h;
    return CC_OK;
}

const char* cc_last_error(const cc_handle* h) {
    if (!h) return "null handle";
    return h->err.c_str();
}

int cc_set_stream(cc_handle* h, void* stream) {
    if (!h) return CC_ERR_ARG;
    h->stream = stream ? (cudaStream_t)stream : h->own;
    return CC_OK;
}

int cc_synchronize(cc_handle* h) {
    if (!h) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, cudaGetErrorString(e));
    return CC_OK;
}

int cc_set_profiling(cc_handle* h, int on) {
    if (!h) return CC_ERR_ARG;
    h->profiling = on != 0;
    return CC_OK;
}

int cc_get_perf(cc_handle* h, cc_perf* out) {
    if (!h || !out) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = h->collect();
    if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, cudaGetErrorString(e));
    *out = h->perf;
    return CC_OK;
}

int cc_reset_perf(cc_handle* h) {
    if (!h) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    cudaError_t e = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = h->collect();
    if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, cudaGetErrorString(e));
    h->perf = cc_perf{};
    return CC_OK;
}

int cc_mhd2d_upload(cc_handle* h, const double* rho, const double* mx, const double* my, const double* mz,
                    const double* E, const double* Bz, const double* Bx_f, const double* By_f) {
    Mhd2dBase* m = m2(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const double* f[8] = {rho, mx, my, mz, E, Bz, Bx_f, By_f};
    return m->upload(f);
}

int cc_mhd2d_download(cc_handle* h, double* rho, double* mx, double* my, double* mz, double* E, double* Bz,
                      double* Bx_f, double* By_f) {
    Mhd2dBase* m = m2(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    double* f[8] = {rho, mx, my, mz, E, Bz, Bx_f, By_f};
    return m->download(f);
}

int cc_mhd2d_compute_gravity(cc_handle* h, double* gx, double* gy) {
    Mhd2dBase* m = m2(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->gravity(gx, gy);
}

int cc_mhd2d_compute_dt(cc_handle* h, double* dt) {
    Mhd2dBase* m = m2(h);
    if (!m || !dt) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->compute_dt(dt);
}

int cc_mhd2d_rk2_step(cc_handle* h, const double* gx, const double* gy, double dt) {
    Mhd2dBase* m = m2(h);
    if (!m) return CC_ERR_ARG;
    if (!std::isfinite(dt) || dt < 0.0) return fail(h, CC_ERR_NONFINITE, "dt not finite or negative");
    if (int r = set_dev(h)) return r;
    return m->rk2_step(gx, gy, dt);
}

int cc_mhd2d_set_stage_kernel(cc_handle* h, int kind, int seg_rows) {
    Mhd2dBase* m = m2(h);
    if (!m) return CC_ERR_ARG;
    return m->set_stage_kernel(kind, seg_rows);
}

int cc_mhd2d_advance(cc_handle* h, int nsteps, double* t) {
    Mhd2dBase* m = m2(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->advance(nsteps, t);
}

int cc_mhd2d_diagnostics(cc_handle* h, cc_diag* d) {
    Mhd2dBase* m = m2(h);
    if (!m || !d) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->diagnostics(d);
}

int cc_mhd2d_derived(cc_handle* h, double* const* out) {
    Mhd2dBase* m = m2(h);
    if (!m || !out) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->derived(out);
}

int cc_mhd2d_checkpoint_save(cc_handle* h, const char* path) {
    Mhd2dBase* m = m2(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_mhd2d_params& p = m->params();
    std::vector<std::vector<double>> f;
    for (size_t n : ck_sizes(p)) f.emplace_back(n);
    double* fp[8];
    for (int k = 0; k < 8; k++) fp[k] = f[k].data();
    if (int r = m->download(fp)) return r;
    double t = 0.0;
    long long steps = 0;
    if (int r = m->get_clock(&t, &steps)) return r;
    std::vector<unsigned char> b;
    ck_put(b, CK_MAGIC, 8);
    const uint32_t ver = CK_VERSION, prec = (uint32_t)p.precision;
    const int32_t nx = p.Nx, ny = p.Ny;
    const uint64_t pb = sizeof(cc_mhd2d_params);
    ck_put(b, &ver, 4); ck_put(b, &prec, 4); ck_put(b, &nx, 4); ck_put(b, &ny, 4);
    ck_put(b, &pb, 8); ck_put(b, &p, sizeof(p));
    ck_put(b, &t, 8); ck_put(b, &steps, 8);
    for (int k = 0; k < 8; k++) ck_put(b, f[k].data(), sizeof(double) * f[k].size());
    const uint64_t sum = ck_fnv1a(b.data(), b.size());
    ck_put(b, &sum, 8);
    FILE* fo = std::fopen(path, "wb");
    if (!fo) return fail(h, CC_ERR_IO, std::string("cannot open for writing: ") + path);
    const size_t w = std::fwrite(b.data(), 1, b.size(), fo);
    const int cl = std::fclose(fo);
    if (w != b.size() || cl != 0) return fail(h, CC_ERR_IO, std::string("short write: ") + path);
    return CC_OK;
}

int cc_mhd2d_checkpoint_load(cc_handle* h, const char* path) {
    Mhd2dBase* m = m2(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_mhd2d_params& p = m->params();
    FILE* fi = std::fopen(path, "rb");
    if (!fi) return fail(h, CC_ERR_IO, std::string("cannot open for reading: ") + path);
    std::vector<unsigned char> b;
    unsigned char chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof(chunk), fi)) > 0) b.insert(b.end(), chunk, chunk + got);
    const bool rerr = std::ferror(fi) != 0;
    std::fclose(fi);
    if (rerr) return fail(h, CC_ERR_IO, std::string("read error: ") + path);
    const size_t head = 8 + 4 * 4 + 8;
    if (b.size() < head + 8 || std::memcmp(b.data(), CK_MAGIC, 8) != 0)
        return fail(h, CC_ERR_ARG, "not a 2D MHD checkpoint (magic)");
    uint64_t sum = 0;
    std::memcpy(&sum, b.data() + b.size() - 8, 8);
    if (sum != ck_fnv1a(b.data(), b.size() - 8)) return fail(h, CC_ERR_ARG, "checkpoint checksum mismatch");
    size_t off = 8;
    uint32_t ver = 0, prec = 0;
    int32_t nx = 0, ny = 0;
    uint64_t pb = 0;
    ck_get(b, off, &ver, 4); ck_get(b, off, &prec, 4); ck_get(b, off, &nx, 4); ck_get(b, off, &ny, 4);
    ck_get(b, off, &pb, 8);
    if (ver != CK_VERSION || pb != sizeof(cc_mhd2d_params)) return fail(h, CC_ERR_ARG, "checkpoint version mismatch");
    cc_mhd2d_params q;
    ck_get(b, off, &q, sizeof(q));
    if (nx != p.Nx || ny != p.Ny || (int)prec != p.precision || q.x0 != p.x0 || q.x1 != p.x1 || q.y0 != p.y0 ||
        q.y1 != p.y1 || q.periodic_x != p.periodic_x || q.periodic_y != p.periodic_y)
        return fail(h, CC_ERR_ARG, "checkpoint grid, domain, boundaries or precision differ from the handle's");
    double t = 0.0;
    long long steps = 0;
    ck_get(b, off, &t, 8); ck_get(b, off, &steps, 8);
    const std::vector<size_t> sz = ck_sizes(p);
    size_t need = off + 8;
    for (size_t n : sz) need += sizeof(double) * n;
    if (need != b.size()) return fail(h, CC_ERR_ARG, "checkpoint size does not match its grid");
    std::vector<std::vector<double>> f;
    for (size_t n : sz) {
        f.emplace_back(n);
        ck_get(b, off, f.back().data(), sizeof(double) * n);
    }
    const double* fp[8];
    for (int k = 0; k < 8; k++) fp[k] = f[k].data();
    if (int r = m->upload(fp)) return r;
    return m->set_clock(t, steps);
}

}  // extern "C"
