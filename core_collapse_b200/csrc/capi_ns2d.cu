// C ABI of the 2D Navier-Stokes + FFT self-gravity step
// (navier_stokes_2d_hllc_poisson.cpp, cited NS:<line>).
//
// Per step (NS:758-791): CFL, minimum and floored-sum partials of U;
// dt = min(cfl h / max speed, cfl_visc h^2 / (mu / rho_min)) (NS:521-546),
// clamped to t_end (NS:759-760); Poisson(U) -> phi; stage 1: k1 = rhs(U),
// U1 = U + dt k1; Poisson(U1) -> phi; stage 2: U = U + dt/2 (k1 + rhs(U1));
// t += dt.  The Poisson solve is the spectral one of the 2D MHD handle
// (reference FFT order in FP64, the FP32 radix-16 transform in FP32) on the
// floored density of the stage input (NS:372-383).
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "checkpoint.h"
#include "fft_tables.h"
#include "handle.h"
#include "ns2d_launch.h"

using namespace ccb;

namespace {

bool ns_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
int ns_log2(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }

struct Ns2dBase {
    virtual ~Ns2dBase() {}
    virtual int init() = 0;
    virtual int upload(const double* const* f) = 0;
    virtual int download(double* const* f) = 0;
    virtual int compute_dt(double* dt) = 0;
    virtual int gravity(double* phi, double* gx, double* gy) = 0;
    virtual int rhs(double* const* dU) = 0;
    virtual int rk2_step(double dt) = 0;
    virtual int advance(int nsteps, double* t) = 0;
    virtual int diagnostics(cc_diag* d) = 0;
    virtual int derived(double* const* out) = 0;
    virtual int get_clock(double* t, long long* steps) = 0;
    virtual int set_clock(double t, long long steps) = 0;
    virtual const cc_ns2d_params& params() const = 0;
};

template <class T> struct Ns2d : Ns2dBase {
    cc_handle* h;
    cc_ns2d_params p;
    NSConst<T> c{};
    int P = 0;
    size_t plane = 0;
    void* block = nullptr;            // U, U1, K: 12 planes
    NSFields<T> U{}, U1{}, K{};
    T* phi = nullptr;
    T* rhof = nullptr;                // floored density of an uploaded state (see raw_low)
    T* g2 = nullptr;                  // gx, gy planes of cc_ns2d_compute_gravity
    Cplx<T>* fftA = nullptr;
    Cplx<T>* tw[4] = {nullptr, nullptr, nullptr, nullptr};   // FP64: radix-2 twiddles; FP32: roots in [0], [2]
    double *staging = nullptr, *spd_part = nullptr, *rmin_part = nullptr, *rho_part = nullptr;
    double *diag_part = nullptr, *scal = nullptr, *derived_dev = nullptr;
    long long* steps_dev = nullptr;
    int* iflags = nullptr;            // active
    bool loaded = false;
    // The state's density may lie below floor_rho only as uploaded: every step
    // floors it (NS:770, 780).  While this is set the stage-1 Poisson input is
    // a floored copy, and advance() runs eagerly.
    bool raw_low = false;
    cudaGraphExec_t graph1 = nullptr;
    cudaStream_t graph_stream = nullptr;
    cc_perf graph_delta{};

    Ns2d(cc_handle* hh, const cc_ns2d_params& pp) : h(hh), p(pp) {}
    cc_handle* this_handle() { return h; }
    cudaStream_t st() const { return h->stream; }
    double* dt_dev() { return scal; }
    double* t_dev() { return scal + 1; }
    double* zero_dev() { return scal + 2; }
    int* active() { return iflags; }
    void count(int n) { h->perf.kernel_launches += n; }

    ~Ns2d() override {
        if (graph1) cudaGraphExecDestroy(graph1);
        void* ptrs[] = {block, phi, rhof, g2, fftA, tw[0], tw[1], tw[2], tw[3], staging, spd_part, rmin_part,
                        rho_part, diag_part, scal, derived_dev, steps_dev, iflags};
        for (void* q : ptrs)
            if (q) cudaFree(q);
    }

    int init() override {
        const int nx = p.Nx, ny = p.Ny;
        const double Lx = p.x1 - p.x0, Ly = p.y1 - p.y0;
        const double dx = Lx / nx, dy = Ly / ny;   // Grid2D (NS:95-111)
        c.gamma = (T)p.gamma;
        c.gm1 = (T)(p.gamma - 1.0);
        c.floor_rho = (T)p.floor_rho; c.floor_P = (T)p.floor_P;
        c.mu = (T)p.mu;
        c.idx1 = (T)(1.0 / dx); c.idy1 = (T)(1.0 / dy);
        c.idx2 = (T)(1.0 / (2.0 * dx)); c.idy2 = (T)(1.0 / (2.0 * dy));
        c.nx = nx; c.ny = ny;
        P = ((nx + 31) / 32) * 32;
        c.pitch = P;
        c.viscous = (p.viscosity_on && p.mu > 0.0) ? 1 : 0;
        c.gravity_on = p.gravity_on ? 1 : 0;
        plane = (size_t)P * ny;
        if (p.gravity_on) {   // the spectral solve's limits (NS:614-617 and the FFT kernels' shared memory)
            if (!ns_pow2(nx) || !ns_pow2(ny) || nx < 4 || ny < 4)
                return fail(h, CC_ERR_UNSUPPORTED, "FFT Poisson needs power-of-two Nx, Ny >= 4");
            if ((size_t)nx * sizeof(Cplx<T>) > 200 * 1024 ||
                (size_t)ny * sizeof(Cplx<T>) * (sizeof(T) == 8 ? 2 : 4) > 200 * 1024)
                return fail(h, CC_ERR_UNSUPPORTED, "FFT line does not fit in shared memory");
            if (sizeof(T) == 4 && (nx > FFT32_MAXN || ny > FFT32_MAXN))
                return fail(h, CC_ERR_UNSUPPORTED, "FP32 FFT Poisson supports Nx, Ny <= 8192");
        }
        CC_CUDA(NSLaunch<T>::prepare());
        CC_CUDA(M2Launch<T>::prepare(nx, ny));
        CC_CUDA(cudaMalloc(&block, sizeof(T) * plane * 12));
        CC_CUDA(cudaMemsetAsync(block, 0, sizeof(T) * plane * 12, st()));
        T* b = reinterpret_cast<T*>(block);
        U = NSFields<T>{b, b + plane, b + 2 * plane, b + 3 * plane};
        U1 = NSFields<T>{b + 4 * plane, b + 5 * plane, b + 6 * plane, b + 7 * plane};
        K = NSFields<T>{b + 8 * plane, b + 9 * plane, b + 10 * plane, b + 11 * plane};
        CC_CUDA(cudaMalloc(&phi, sizeof(T) * plane));
        CC_CUDA(cudaMemsetAsync(phi, 0, sizeof(T) * plane, st()));
        if (p.gravity_on) {
            if constexpr (sizeof(T) == 4) {
                CC_CUDA(cudaMalloc(&fftA, sizeof(Cplx<T>) * (size_t)fft32_half_lines(nx) * ny));
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
                    const std::vector<double> t = twiddle_table(ns[k], k & 1);
                    CC_CUDA(cudaMalloc(&tw[k], sizeof(double) * t.size()));
                    CC_CUDA(cudaMemcpyAsync(tw[k], t.data(), sizeof(double) * t.size(), cudaMemcpyHostToDevice, st()));
                }
            }
        }
        CC_CUDA(cudaMalloc(&staging, sizeof(double) * (size_t)nx * ny));
        CC_CUDA(cudaMalloc(&spd_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&rmin_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&rho_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&diag_part, sizeof(double) * RED_BLOCKS * 5));
        CC_CUDA(cudaMalloc(&scal, sizeof(double) * 4));
        CC_CUDA(cudaMemsetAsync(scal, 0, sizeof(double) * 4, st()));
        CC_CUDA(cudaMalloc(&steps_dev, sizeof(long long)));
        CC_CUDA(cudaMemsetAsync(steps_dev, 0, sizeof(long long), st()));
        CC_CUDA(cudaMalloc(&iflags, sizeof(int) * 4));
        const int init_flags[4] = {1, 0, 0, 0};
        CC_CUDA(cudaMemcpyAsync(iflags, init_flags, sizeof(init_flags), cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    T* field(const NSFields<T>& f, int k) const {
        T* a[4] = {f.d, f.mx, f.my, f.E};
        return a[k];
    }

    int upload(const double* const* f) override {
        const size_t n = (size_t)p.Nx * p.Ny;
        for (int k = 0; k < 4; k++)
            if (!f[k]) return fail(h, CC_ERR_ARG, "null state array");
        bool low = false;   // any density below the floor (or NaN) in the state's precision
        for (size_t q = 0; q < n && !low; q++) low = !((T)f[0][q] >= (T)p.floor_rho);
        for (int k = 0; k < 4; k++) {
            CC_CUDA(cudaMemcpyAsync(staging, f[k], sizeof(double) * n, cudaMemcpyHostToDevice, st()));
            CC_CUDA(M2Launch<T>::pack_in(staging, field(U, k), p.Nx, p.Ny, P, st()));
            count(1);
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        if (low && !rhof) CC_CUDA(cudaMalloc(&rhof, sizeof(T) * plane));
        raw_low = low;
        loaded = true;
        return CC_OK;
    }

    int download(double* const* f) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        return download_fields(U, f);
    }

    int download_fields(const NSFields<T>& s, double* const* f) {
        for (int k = 0; k < 4; k++) {
            if (!f[k]) continue;
            CC_CUDA(M2Launch<T>::pack_out(field(s, k), staging, p.Nx, p.Ny, P, st()));
            count(1);
            CC_CUDA(cudaMemcpyAsync(f[k], staging, sizeof(double) * (size_t)p.Nx * p.Ny, cudaMemcpyDeviceToHost, st()));
            CC_CUDA(cudaStreamSynchronize(st()));
        }
        return CC_OK;
    }

    // spectral Poisson on a density plane whose (floored) sum is in rho_part -> phi
    int solve(const T* rho) {
        h->perf.poisson_solves += 1;
        const int nx = p.Nx, ny = p.Ny;
        if constexpr (sizeof(T) == 4)
            CC_CUDA(M2Launch<T>::fft32_solve(rho, P, rho_part, nx, ny, reinterpret_cast<const float2*>(tw[0]),
                                             reinterpret_cast<const float2*>(tw[2]), p.x1 - p.x0, p.y1 - p.y0, p.G,
                                             reinterpret_cast<float2*>(fftA), phi, active(), st()));
        else
            CC_CUDA(M2Launch<T>::fft_solve(rho, P, rho_part, nx, ny, ns_log2(nx), ns_log2(ny), tw[0], tw[1], tw[2],
                                           tw[3], p.x1 - p.x0, p.y1 - p.y0, p.G, fftA, phi, active(), st()));
        count(3);
        return CC_OK;
    }

    // Poisson input of U: its density, or the floored copy while raw_low
    const T* u_density() {
        return raw_low ? rhof : U.d;
    }
    int floor_u() {
        if (!raw_low) return CC_OK;
        CC_CUDA(NSLaunch<T>::floor_copy(c, U.d, rhof, active(), st()));
        count(1);
        return CC_OK;
    }

    NSDtSpec dtspec(bool clamp) const {
        const double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
        NSDtSpec d;
        d.cfl = p.cfl; d.hmin = vmin(dx, dy); d.mu = p.mu; d.cfl_visc = p.cfl_visc; d.floor_rho = p.floor_rho;
        d.t_end = p.t_end; d.viscous = c.viscous; d.clamp_to_end = clamp ? 1 : 0;
        return d;
    }

    int set_active() {
        const int one = 1;
        CC_CUDA(cudaMemcpyAsync(iflags, &one, sizeof(int), cudaMemcpyHostToDevice, st()));
        return CC_OK;
    }

    int compute_dt(double* dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        CC_CUDA(NSLaunch<T>::speeds(c, U, spd_part, rmin_part, rho_part, st()));
        CC_CUDA(launch_ns_dt(spd_part, rmin_part, dtspec(false), dt_dev(), t_dev(), active(), st()));
        count(2);
        CC_CUDA(cudaMemcpyAsync(dt, dt_dev(), sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    // phi of U's density (NS:379-383); rho_part of U is computed here
    int potential_of_u() {
        CC_CUDA(NSLaunch<T>::speeds(c, U, spd_part, rmin_part, rho_part, st()));
        count(1);
        if (int r = floor_u()) return r;
        return solve(u_density());
    }

    int gravity(double* phi_out, double* gx, double* gy) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        if (int r = set_active()) return r;
        if (!g2) CC_CUDA(cudaMalloc(&g2, sizeof(T) * plane * 2));
        if (p.gravity_on) {
            if (int r = potential_of_u()) return r;
            CC_CUDA(NSLaunch<T>::gravity(c, phi, g2, g2 + plane, st()));
            count(1);
        } else {
            CC_CUDA(cudaMemsetAsync(phi, 0, sizeof(T) * plane, st()));
            CC_CUDA(cudaMemsetAsync(g2, 0, sizeof(T) * plane * 2, st()));
        }
        const T* src[3] = {phi, g2, g2 + plane};
        double* dst[3] = {phi_out, gx, gy};
        for (int k = 0; k < 3; k++) {
            if (!dst[k]) continue;
            CC_CUDA(M2Launch<T>::pack_out(src[k], staging, p.Nx, p.Ny, P, st()));
            count(1);
            CC_CUDA(cudaMemcpyAsync(dst[k], staging, sizeof(double) * (size_t)p.Nx * p.Ny, cudaMemcpyDeviceToHost, st()));
            CC_CUDA(cudaStreamSynchronize(st()));
        }
        return CC_OK;
    }

    // compute_rhs (NS:363-518): the stage-1 kernel with dt = 0 writes k1 = rhs(U) into K
    int rhs(double* const* dU) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        if (int r = set_active()) return r;
        if (p.gravity_on)
            if (int r = potential_of_u()) return r;
        CC_CUDA(NSLaunch<T>::stage(c, U, U, K, U1, false, phi, zero_dev(), active(), st()));
        count(1);
        return download_fields(K, dU);
    }

    // the Heun step (NS:762-781) with dt in dt_dev; each rhs solves Poisson itself (NS:379-383)
    int step_body() {
        if (p.gravity_on) {   // rho_part of U comes from speeds() or from here
            if (int r = floor_u()) return r;
            if (int r = solve(u_density())) return r;
        }
        CC_CUDA(NSLaunch<T>::stage(c, U, U, K, U1, false, phi, dt_dev(), active(), st()));
        count(1);
        if (p.gravity_on) {
            CC_CUDA(NSLaunch<T>::rho_sum(c, U1.d, rho_part, st()));
            count(1);
            if (int r = solve(U1.d)) return r;
        }
        CC_CUDA(NSLaunch<T>::stage(c, U, U1, K, U, true, phi, dt_dev(), active(), st()));
        count(1);
        h->perf.steps += 1;
        return CC_OK;
    }

    int rk2_step(double dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        if (int r = set_active()) return r;
        CC_CUDA(launch_set_scalar(dt_dev(), dt, st()));
        count(1);
        if (p.gravity_on) {
            CC_CUDA(NSLaunch<T>::speeds(c, U, spd_part, rmin_part, rho_part, st()));
            count(1);
        }
        if (int r = step_body()) return r;
        CC_CUDA(cudaStreamSynchronize(st()));
        raw_low = false;
        return CC_OK;
    }

    int device_step() {
        CC_CUDA(NSLaunch<T>::speeds(c, U, spd_part, rmin_part, rho_part, st()));
        CC_CUDA(launch_ns_dt(spd_part, rmin_part, dtspec(true), dt_dev(), t_dev(), active(), st()));
        count(2);
        if (int r = step_body()) return r;
        CC_CUDA(launch_clock(t_dev(), dt_dev(), active(), steps_dev, st()));
        count(1);
        return CC_OK;
    }

    int advance(int nsteps, double* t) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        if (nsteps < 0) return fail(h, CC_ERR_ARG, "nsteps < 0");
        if (t) {
            CC_CUDA(launch_set_scalar(t_dev(), *t, st()));
            count(1);
        }
        int k = 0;
        while (raw_low && k < nsteps) {   // eager until a step has floored the uploaded density
            long long before = 0, after = 0;
            CC_CUDA(cudaMemcpyAsync(&before, steps_dev, sizeof(before), cudaMemcpyDeviceToHost, st()));
            if (int r = device_step()) return r;
            CC_CUDA(cudaMemcpyAsync(&after, steps_dev, sizeof(after), cudaMemcpyDeviceToHost, st()));
            CC_CUDA(cudaStreamSynchronize(st()));
            if (after == before) break;   // past t_end: nothing more runs
            raw_low = false;
            k++;
        }
        nsteps = raw_low ? 0 : nsteps - k;
        if (!h->profiling && nsteps >= 1) {
            if (!graph1 || graph_stream != st()) {
                if (graph1) { cudaGraphExecDestroy(graph1); graph1 = nullptr; }
                const cc_perf before = h->perf;
                cudaGraph_t g = nullptr;
                CC_CUDA(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
                int rr = device_step();
                cudaError_t e = cudaStreamEndCapture(st(), &g);
                graph_delta.kernel_launches = h->perf.kernel_launches - before.kernel_launches;
                graph_delta.steps = h->perf.steps - before.steps;
                graph_delta.poisson_solves = h->perf.poisson_solves - before.poisson_solves;
                h->perf = before;
                if (rr) { if (g) cudaGraphDestroy(g); return rr; }
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
                e = cudaGraphInstantiate(&graph1, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
                graph_stream = st();
            }
            for (int s = 0; s < nsteps; s++) {
                CC_CUDA(cudaGraphLaunch(graph1, st()));
                h->perf.kernel_launches += graph_delta.kernel_launches;
                h->perf.steps += graph_delta.steps;
                h->perf.poisson_solves += graph_delta.poisson_solves;
            }
        } else {
            for (int s = 0; s < nsteps; s++)
                if (int r = device_step()) return r;
        }
        if (t) CC_CUDA(cudaMemcpyAsync(t, t_dev(), sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int derived(double* const* out) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        const size_t n = (size_t)p.Nx * p.Ny;
        if (int r = set_active()) return r;
        if (!derived_dev) CC_CUDA(cudaMalloc(&derived_dev, sizeof(double) * n * 8));
        if (p.gravity_on)   // the store's Phi (NS:735-745)
            if (int r = potential_of_u()) return r;
        CC_CUDA(NSLaunch<T>::derived(c, U, p.gravity_on ? phi : nullptr, derived_dev, st()));
        count(1);
        for (int k = 0; k < 8; k++)
            if (out[k])
                CC_CUDA(cudaMemcpyAsync(out[k], derived_dev + k * n, sizeof(double) * n, cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int get_clock(double* t, long long* steps) override {
        CC_CUDA(cudaMemcpyAsync(t, t_dev(), sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaMemcpyAsync(steps, steps_dev, sizeof(long long), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int set_clock(double t, long long steps) override {
        CC_CUDA(launch_set_scalar(t_dev(), t, st()));
        CC_CUDA(cudaMemcpyAsync(steps_dev, &steps, sizeof(long long), cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    const cc_ns2d_params& params() const override { return p; }

    int diagnostics(cc_diag* d) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        CC_CUDA(NSLaunch<T>::diag(c, U, diag_part, st()));
        count(1);
        std::vector<double> part(RED_BLOCKS * 5);
        CC_CUDA(cudaMemcpyAsync(part.data(), diag_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st()));
        double sc[4];
        CC_CUDA(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st()));
        long long steps = 0;
        CC_CUDA(cudaMemcpyAsync(&steps, steps_dev, sizeof(steps), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        double s[4] = {0, 0, 0, 0}, nonf = 0.0;
        for (int m = 0; m < 4; m++)
            for (int b = 0; b < RED_BLOCKS; b++) s[m] += part[m * RED_BLOCKS + b];
        for (int b = 0; b < RED_BLOCKS; b++) nonf = std::fmax(nonf, part[4 * RED_BLOCKS + b]);
        const double dV = ((p.x1 - p.x0) / p.Nx) * ((p.y1 - p.y0) / p.Ny);
        std::memset(d, 0, sizeof(*d));
        d->mass = s[0] * dV; d->mom_x = s[1] * dV; d->mom_y = s[2] * dV; d->energy = s[3] * dV;
        d->t = sc[1]; d->dt_last = sc[0]; d->steps = steps;
        d->nonfinite = nonf > 0.0 ? 1 : 0;
        return CC_OK;
    }
};

struct Ns2dHandle : cc_handle {
    std::unique_ptr<Ns2dBase> impl;
};

Ns2dBase* ns(cc_handle* h) {
    if (!h || h->kind != KIND_NS2D) return nullptr;
    return static_cast<Ns2dHandle*>(h)->impl.get();
}

}  // namespace

extern "C" {

void cc_ns2d_params_default(cc_ns2d_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma = 1.4; p->cfl = 0.35;
    p->x0 = 0.0; p->x1 = 1.0; p->y0 = 0.0; p->y1 = 1.0;
    p->Nx = 128; p->Ny = 128;
    p->t_end = 10.0; p->dt_store = 5e-3;
    p->seed = 42;
    p->floor_rho = 1e-10; p->floor_P = 1e-10;
    p->viscosity_on = 1; p->mu = 1e-6; p->cfl_visc = 0.05;
    p->gravity_on = 1; p->G = 10.0;
    p->precision = CC_FP64;
}

int cc_ns2d_create(const cc_ns2d_params* p, cc_handle** out) {
    if (!p || !out) return CC_ERR_ARG;
    *out = nullptr;
    if (p->Nx < 2 || p->Ny < 2 || !(p->x1 > p->x0) || !(p->y1 > p->y0)) return CC_ERR_ARG;
    if (p->precision != CC_FP64 && p->precision != CC_FP32) return CC_ERR_ARG;
    auto h = std::make_unique<Ns2dHandle>();
    h->kind = KIND_NS2D;
    if (cudaGetDevice(&h->device) != cudaSuccess) return CC_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return CC_ERR_CUDA;
    h->stream = h->own;
    if (p->precision == CC_FP64) h->impl = std::make_unique<Ns2d<double>>(h.get(), *p);
    else h->impl = std::make_unique<Ns2d<float>>(h.get(), *p);
    int r = h->impl->init();
    *out = h.release();
    return r;
}

int cc_ns2d_upload(cc_handle* h, const double* rho, const double* mx, const double* my, const double* E) {
    Ns2dBase* m = ns(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const double* f[4] = {rho, mx, my, E};
    return m->upload(f);
}

int cc_ns2d_download(cc_handle* h, double* rho, double* mx, double* my, double* E) {
    Ns2dBase* m = ns(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    double* f[4] = {rho, mx, my, E};
    return m->download(f);
}

int cc_ns2d_compute_dt(cc_handle* h, double* dt) {
    Ns2dBase* m = ns(h);
    if (!m || !dt) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->compute_dt(dt);
}

int cc_ns2d_compute_gravity(cc_handle* h, double* phi, double* gx, double* gy) {
    Ns2dBase* m = ns(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->gravity(phi, gx, gy);
}

int cc_ns2d_compute_rhs(cc_handle* h, double* const* dU) {
    Ns2dBase* m = ns(h);
    if (!m || !dU) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->rhs(dU);
}

int cc_ns2d_rk2_step(cc_handle* h, double dt) {
    Ns2dBase* m = ns(h);
    if (!m) return CC_ERR_ARG;
    if (!std::isfinite(dt) || dt <= 0.0) return fail(h, CC_ERR_NONFINITE, "dt not finite or not positive");
    if (int r = set_dev(h)) return r;
    return m->rk2_step(dt);
}

int cc_ns2d_advance(cc_handle* h, int nsteps, double* t) {
    Ns2dBase* m = ns(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->advance(nsteps, t);
}

int cc_ns2d_diagnostics(cc_handle* h, cc_diag* d) {
    Ns2dBase* m = ns(h);
    if (!m || !d) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->diagnostics(d);
}

int cc_ns2d_derived(cc_handle* h, double* const* out) {
    Ns2dBase* m = ns(h);
    if (!m || !out) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->derived(out);
}

// restart files (checkpoint.h): state {rho, mx, my, E} and the clock
int cc_ns2d_checkpoint_save(cc_handle* h, const char* path) {
    Ns2dBase* m = ns(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_ns2d_params& p = m->params();
    const size_t n = (size_t)p.Nx * p.Ny;
    std::vector<std::vector<double>> f(4, std::vector<double>(n));
    double* fp[4] = {f[0].data(), f[1].data(), f[2].data(), f[3].data()};
    if (int r = m->download(fp)) return r;
    CkMeta meta;
    meta.precision = (uint32_t)p.precision;
    meta.n[0] = p.Nx; meta.n[1] = p.Ny;
    if (int r = m->get_clock(&meta.t, &meta.steps)) return r;
    std::string err;
    if (int r = ck3_save(path, "CCNS2CK1", meta, &p, sizeof(p), f, err)) return fail(h, r, err);
    return CC_OK;
}

int cc_ns2d_checkpoint_load(cc_handle* h, const char* path) {
    Ns2dBase* m = ns(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_ns2d_params& p = m->params();
    CkMeta meta;
    cc_ns2d_params q;
    std::vector<std::vector<double>> f;
    std::string err;
    auto sizes = [](const int32_t* n) { return std::vector<size_t>(4, (size_t)n[0] * n[1]); };
    if (int r = ck3_load(path, "CCNS2CK1", meta, &q, sizeof(q), sizes, f, err)) return fail(h, r, err);
    if (meta.n[0] != p.Nx || meta.n[1] != p.Ny || (int)meta.precision != p.precision || q.x0 != p.x0 ||
        q.x1 != p.x1 || q.y0 != p.y0 || q.y1 != p.y1)
        return fail(h, CC_ERR_ARG, "checkpoint grid, domain or precision differ from the handle's");
    const double* fp[4] = {f[0].data(), f[1].data(), f[2].data(), f[3].data()};
    if (int r = m->upload(fp)) return r;
    return m->set_clock(meta.t, meta.steps);
}

}  // extern "C"
