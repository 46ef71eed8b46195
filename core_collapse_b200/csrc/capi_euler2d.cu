// C ABI of the 2D Euler + self-gravity HLLC step (euler2d_gravity_hllc.cpp).
//
// Per step (EH:697-706, 529-550): CFL partials and floored-density sums of U;
// dt = cfl min(dx,dy) / max speed, a non-finite or non-positive dt stops the
// loop with CC_ERR_NONFINITE (EH:699-702), clamp to t_end;
// Poisson(U) -> phi; stage 1: U1 = floors(U + dt rhs(U));
// Poisson(U1) -> phi; stage 2: U = floors(0.5 U + 0.5 (U1 + dt rhs(U1)));
// t += dt.  The Poisson solve floors the density and always wraps (EH:300-317).
#include <algorithm>
#include <utility>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "checkpoint.h"
#include "euler2d_launch.h"
#include "handle.h"

using namespace ccb;

namespace {

struct Euler2dBase {
    virtual ~Euler2dBase() {}
    virtual int init() = 0;
    virtual int upload(const double* const* f) = 0;
    virtual int download(double* const* f) = 0;
    virtual int compute_dt(double* dt) = 0;
    virtual int gravity(double* gx, double* gy) = 0;
    virtual int rk2_step(double dt) = 0;
    virtual int advance(int nsteps, double* t) = 0;
    virtual int diagnostics(cc_diag* d) = 0;
    virtual int derived(double* const* out) = 0;
    virtual int get_clock(double* t, long long* steps) = 0;
    virtual int set_clock(double t, long long steps) = 0;
    virtual const cc_euler2d_params& params() const = 0;
};

template <class T> struct Euler2d : Euler2dBase {
    cc_handle* h;
    cc_euler2d_params p;
    EHConst<T> c{};
    int P = 0;
    size_t plane = 0;
    void* block = nullptr;
    EHFields<T> U{}, U1{};
    T* phi = nullptr;
    T* g2[2] = {nullptr, nullptr};
    double *rhs = nullptr, *sphi = nullptr, *sor_part = nullptr, *sor_part2 = nullptr;
    double *staging = nullptr, *spd_part = nullptr, *rho_part = nullptr, *diag_part = nullptr, *scal = nullptr;
    unsigned int* bar = nullptr;
    long long* steps_dev = nullptr;
    int* iflags = nullptr;   // active, barrier error, SOR sweeps, bad dt
    double* derived_dev = nullptr;   // 3 planes of Nx*Ny, allocated at the first cc_euler2d_derived
    // enclosed-mass gravity: cells in radius order, each one's group end, scan scratch
    int* enc_order = nullptr;
    int* enc_gend = nullptr;
    double* enc_cum = nullptr;
    double* enc_blk = nullptr;
    bool enclosed() const { return p.gravity_on && p.poisson_kind == CC_GRAVITY_ENCLOSED; }
    bool shells() const { return p.gravity_on && p.poisson_kind == CC_GRAVITY_SHELLS; }
    bool radial() const { return enclosed() || shells(); }   // gravity as arrays, no Poisson solve
    double* shl_geo = nullptr;   // shells: per sorted cell rx, ry, (r^2 + softening^2)^(3/2)
    bool loaded = false;
    cudaGraphExec_t graph1 = nullptr;
    cudaStream_t graph_stream = nullptr;
    cc_perf graph_delta{};

    Euler2d(cc_handle* hh, const cc_euler2d_params& pp) : h(hh), p(pp) {}
    cc_handle* this_handle() { return h; }
    cudaStream_t st() const { return h->stream; }
    double* dt_dev() { return scal; }
    double* t_dev() { return scal + 1; }
    double* res_dev() { return scal + 2; }
    int* active() { return iflags; }
    void count(int n) { h->perf.kernel_launches += n; }

    ~Euler2d() override {
        if (graph1) cudaGraphExecDestroy(graph1);
        void* ptrs[] = {block, phi, g2[0], g2[1], rhs, sphi, sor_part, sor_part2, staging, spd_part, rho_part,
                        diag_part, scal, bar, steps_dev, iflags, derived_dev, enc_order, enc_gend, enc_cum,
                        enc_blk, shl_geo};
        for (void* q : ptrs)
            if (q) cudaFree(q);
    }

    int init() override {
        const int nx = p.Nx, ny = p.Ny;
        const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
        c.gamma = (T)p.gamma; c.gm1 = (T)p.gamma - (T)1.0;
        c.floor_rho = (T)p.floor_rho; c.floor_P = (T)p.floor_P;
        c.dx = (T)dx; c.dy = (T)dy; c.two_dx = (T)(2.0 * dx); c.two_dy = (T)(2.0 * dy);
        c.nx = nx; c.ny = ny;
        P = ((nx + 1 + 31) / 32) * 32;
        c.pitch = P;
        c.ax = AxisMap{nx, p.periodic_x ? 1 : 0};
        c.ay = AxisMap{ny, p.periodic_y ? 1 : 0};
        c.pax = AxisMap{nx, 1};
        c.pay = AxisMap{ny, 1};
        c.gravity_on = p.gravity_on ? 1 : 0;
        plane = (size_t)P * (ny + 1);
        if (p.gravity_on) {
            if (p.poisson_kind != CC_POISSON_SOR && p.poisson_kind != CC_POISSON_SOR_LEX &&
                p.poisson_kind != CC_GRAVITY_ENCLOSED && p.poisson_kind != CC_GRAVITY_SHELLS)
                return fail(h, CC_ERR_UNSUPPORTED, "the Euler/HLLC solver supports SOR or enclosed-mass gravity");
            if (p.poisson_kind == CC_POISSON_SOR && ((nx & 1) || (ny & 1)))
                return fail(h, CC_ERR_UNSUPPORTED, "red-black SOR needs even Nx and Ny (periodic)");
        }
        CC_CUDA(EHLaunch<T>::prepare());
        CC_CUDA(cudaMalloc(&block, sizeof(T) * plane * 8));
        CC_CUDA(cudaMemsetAsync(block, 0, sizeof(T) * plane * 8, st()));
        T* b = reinterpret_cast<T*>(block);
        U = EHFields<T>{b, b + plane, b + 2 * plane, b + 3 * plane};
        U1 = EHFields<T>{b + 4 * plane, b + 5 * plane, b + 6 * plane, b + 7 * plane};
        CC_CUDA(cudaMalloc(&phi, sizeof(T) * plane));
        CC_CUDA(cudaMemsetAsync(phi, 0, sizeof(T) * plane, st()));
        if (radial()) {   // gravity arrays written by every solve, the radius order built once
            CC_CUDA(cudaMalloc(&g2[0], sizeof(T) * plane));
            CC_CUDA(cudaMalloc(&g2[1], sizeof(T) * plane));
            CC_CUDA(cudaMemsetAsync(g2[0], 0, sizeof(T) * plane, st()));
            CC_CUDA(cudaMemsetAsync(g2[1], 0, sizeof(T) * plane, st()));
            if (int r = enclosed() ? enclosed_setup() : shells_setup()) return r;
        }
        CC_CUDA(cudaMalloc(&staging, sizeof(double) * (size_t)(nx + 1) * (ny + 1)));
        CC_CUDA(cudaMalloc(&spd_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&rho_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&diag_part, sizeof(double) * RED_BLOCKS * 5));
        CC_CUDA(cudaMalloc(&scal, sizeof(double) * 4));
        CC_CUDA(cudaMemsetAsync(scal, 0, sizeof(double) * 4, st()));
        CC_CUDA(cudaMalloc(&steps_dev, sizeof(long long)));
        CC_CUDA(cudaMemsetAsync(steps_dev, 0, sizeof(long long), st()));
        CC_CUDA(cudaMalloc(&iflags, sizeof(int) * 4));
        int init_flags[4] = {1, 0, 0, 0};
        CC_CUDA(cudaMemcpyAsync(iflags, init_flags, sizeof(init_flags), cudaMemcpyHostToDevice, st()));
        if (p.gravity_on) {
            CC_CUDA(cudaMalloc(&rhs, sizeof(double) * (size_t)nx * ny));
            CC_CUDA(cudaMalloc(&sphi, sizeof(double) * (size_t)nx * ny));
            CC_CUDA(cudaMalloc(&sor_part, sizeof(double) * 4096));
            CC_CUDA(cudaMalloc(&sor_part2, sizeof(double) * 4096));
            CC_CUDA(cudaMalloc(&bar, sizeof(unsigned int) * 2));
            CC_CUDA(cudaMemsetAsync(bar, 0, sizeof(unsigned int) * 2, st()));
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    T* field(const EHFields<T>& f, int k) const {
        T* a[4] = {f.rho, f.mx, f.my, f.E};
        return a[k];
    }

    int upload(const double* const* f) override {
        for (int k = 0; k < 4; k++) {
            if (!f[k]) return fail(h, CC_ERR_ARG, "null state array");
            CC_CUDA(cudaMemcpyAsync(staging, f[k], sizeof(double) * (size_t)p.Nx * p.Ny, cudaMemcpyHostToDevice, st()));
            CC_CUDA(M2Launch<T>::pack_in(staging, field(U, k), p.Nx, p.Ny, P, st()));
            count(1);
        }
        loaded = true;
        return CC_OK;
    }

    int download(double* const* f) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        for (int k = 0; k < 4; k++) {
            if (!f[k]) continue;
            CC_CUDA(M2Launch<T>::pack_out(field(U, k), staging, p.Nx, p.Ny, P, st()));
            count(1);
            CC_CUDA(cudaMemcpyAsync(f[k], staging, sizeof(double) * (size_t)p.Nx * p.Ny, cudaMemcpyDeviceToHost, st()));
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    // radius order of the cells and each one's group end (compute_enclosed_mass_gravity,
    // EH:241-269): the radii depend only on the grid, so they are sorted once
    int enclosed_setup() {
        const int nx = p.Nx, ny = p.Ny, n = nx * ny;
        const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
        const double cx = 0.5 * (p.x0 + p.x1), cy = 0.5 * (p.y0 + p.y1);
        std::vector<std::pair<double, int>> cells;
        cells.reserve(n);
        for (int j = 0; j < ny; ++j) {
            const double y = p.y0 + (j + 0.5) * dy;
            for (int i = 0; i < nx; ++i) {
                const double x = p.x0 + (i + 0.5) * dx;
                const double rx = x - cx, ry = y - cy;
                cells.emplace_back(std::sqrt(rx * rx + ry * ry), j * nx + i);
            }
        }
        std::sort(cells.begin(), cells.end(),
                  [](const std::pair<double, int>& a, const std::pair<double, int>& b) { return a.first < b.first; });
        std::vector<int> order(n), gend(n);
        int s = 0;
        while (s < n) {
            const double r0 = cells[s].first;
            int e = s + 1;
            while (e < n && cells[e].first <= r0 + 1e-12) ++e;
            for (int t = s; t < e; ++t) { order[t] = cells[t].second; gend[t] = e; }
            s = e;
        }
        const int nb = (n + ENC_NT - 1) / ENC_NT;
        CC_CUDA(cudaMalloc(&enc_order, sizeof(int) * n));
        CC_CUDA(cudaMalloc(&enc_gend, sizeof(int) * n));
        CC_CUDA(cudaMalloc(&enc_cum, sizeof(double) * n));
        CC_CUDA(cudaMalloc(&enc_blk, sizeof(double) * nb));
        CC_CUDA(cudaMemcpyAsync(enc_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaMemcpyAsync(enc_gend, gend.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaStreamSynchronize(st()));   // the host vectors go out of scope
        return CC_OK;
    }

    // shell-binned enclosed mass (gravity_accel_from_enclosed_mass, gravity_enclosed.h:18-96):
    // the shells depend only on the grid, so each cell's shell is found once and
    // the cells are ordered by shell (index order inside a shell, the reference's
    // deposit order); the scan of enclosed_kernels.cuh then gives M(<shell) at
    // each shell's end.  The geometry factors (the reference's std::pow) are
    // built here on the host, in the sorted order.
    int shells_setup() {
        const int nx = p.Nx, ny = p.Ny, n = nx * ny;
        const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
        auto xof = [&](int i) { return p.x0 + (i + 0.5) * dx; };
        auto yof = [&](int j) { return p.y0 + (j + 0.5) * dy; };
        double rmax = 0.0;
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double ddx = xof(i) - p.xc, ddy = yof(j) - p.yc;
                rmax = std::max(rmax, std::sqrt(ddx * ddx + ddy * ddy));
            }
        rmax = std::max(rmax, 1e-12);
        const int nr = std::max(8, p.Nr_bins);
        const double dr = rmax / (double)nr;
        std::vector<int> bin(n), count(nr + 1, 0);
        for (int j = 0; j < ny; ++j)
            for (int i = 0; i < nx; ++i) {
                const double ddx = xof(i) - p.xc, ddy = yof(j) - p.yc;
                int b = (int)std::floor(std::sqrt(ddx * ddx + ddy * ddy) / dr);
                b = b < 0 ? 0 : (b >= nr ? nr - 1 : b);
                bin[j * nx + i] = b;
                count[b + 1]++;
            }
        for (int b = 0; b < nr; ++b) count[b + 1] += count[b];   // shell starts
        std::vector<int> order(n), gend(n), fill(count.begin(), count.end() - 1);
        for (int k = 0; k < n; ++k) order[fill[bin[k]]++] = k;   // stable: index order inside a shell
        std::vector<double> geo(3 * (size_t)n);
        const double eps2 = p.softening * p.softening;
        for (int t = 0; t < n; ++t) {
            const int k = order[t], i = k % nx, j = k / nx;
            gend[t] = count[bin[k] + 1];
            const double ddx = xof(i) - p.xc, ddy = yof(j) - p.yc;
            geo[t] = ddx;
            geo[n + t] = ddy;
            geo[2 * (size_t)n + t] = std::pow(ddx * ddx + ddy * ddy + eps2, 1.5);
        }
        const int nb = (n + ENC_NT - 1) / ENC_NT;
        CC_CUDA(cudaMalloc(&enc_order, sizeof(int) * n));
        CC_CUDA(cudaMalloc(&enc_gend, sizeof(int) * n));
        CC_CUDA(cudaMalloc(&enc_cum, sizeof(double) * n));
        CC_CUDA(cudaMalloc(&enc_blk, sizeof(double) * nb));
        CC_CUDA(cudaMalloc(&shl_geo, sizeof(double) * geo.size()));
        CC_CUDA(cudaMemcpyAsync(enc_order, order.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaMemcpyAsync(enc_gend, gend.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaMemcpyAsync(shl_geo, geo.data(), sizeof(double) * geo.size(), cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaStreamSynchronize(st()));   // the host vectors go out of scope
        return CC_OK;
    }

    // gravity arrays of the stage kernel: g2 in the enclosed-mass modes, none for SOR (phi)
    const T* gxa() const { return radial() ? g2[0] : nullptr; }
    const T* gya() const { return radial() ? g2[1] : nullptr; }

    // Poisson on a density field whose floored sum is in rho_part -> phi;
    // in the enclosed-mass mode the gravity itself -> g2
    int solve(const T* rho) {
        if (!p.gravity_on) return CC_OK;
        if (shells()) {
            h->perf.poisson_solves += 1;
            const int n = p.Nx * p.Ny;
            const double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
            CC_CUDA(EHLaunch<T>::shells(c, rho, enc_order, enc_gend, n, enc_cum, enc_blk, shl_geo, dx * dy, p.G,
                                        p.floor_rho, g2[0], g2[1], active(), st()));
            count(3);
            return CC_OK;
        }
        if (enclosed()) {
            h->perf.poisson_solves += 1;
            const int nx = p.Nx, ny = p.Ny;
            const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
            CC_CUDA(EHLaunch<T>::enclosed(c, rho, enc_order, enc_gend, nx * ny, enc_cum, enc_blk, p.x0, p.y0, dx,
                                          dy, 0.5 * (p.x0 + p.x1), 0.5 * (p.y0 + p.y1), p.G,
                                          p.softening * p.softening, p.floor_rho, g2[0], g2[1], active(), st()));
            count(3);
            return CC_OK;
        }
        h->perf.poisson_solves += 1;
        const int nx = p.Nx, ny = p.Ny;
        if (p.poisson_kind == CC_POISSON_SOR_LEX) {   // the reference's own order (parity mode)
            const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
            SorLexArgs a;
            a.nx = nx; a.ny = ny; a.pitch = P; a.ax = c.pax; a.ay = c.pay;
            a.idx2 = 1.0 / (dx * dx); a.idy2 = 1.0 / (dy * dy);
            a.denom = 2.0 * (a.idx2 + a.idy2);
            a.omega = p.sor_omega; a.fourpiG = 4.0 * M_PI * p.G; a.tol = p.sor_tol; a.max_iter = p.sor_max_iter;
            a.floor_rho = p.floor_rho;
            a.rhs = rhs; a.phi = sphi; a.iters_out = iflags + 2; a.res_out = res_dev(); a.active = active();
            CC_CUDA(launch_sor_lex<T>(a, rho, st()));
            CC_CUDA(M2Launch<T>::phi_to_field(sphi, nx, ny, phi, P, active(), st()));
            count(2);
            return CC_OK;
        }
        CC_CUDA(M2Launch<T>::sor_rhs(rho, nx, ny, P, rho_part, 4.0 * M_PI * p.G, p.floor_rho, rhs, active(), st()));
        const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny;
        SorArgs a;
        a.nx = nx; a.ny = ny; a.ax = c.pax; a.ay = c.pay;
        a.idx2 = 1.0 / (dx * dx); a.idy2 = 1.0 / (dy * dy);
        a.denom = 2.0 * (a.idx2 + a.idy2);
        a.omega = p.sor_omega; a.tol = p.sor_tol; a.max_iter = p.sor_max_iter;
        a.rhs = rhs; a.phi = sphi; a.part = sor_part; a.part2 = sor_part2;
        a.bar = GridBarrier{bar, bar + 1, iflags + 1};
        a.iters_out = iflags + 2; a.res_out = res_dev(); a.active = active();
        int nb = 0;
        CC_CUDA(launch_sor(a, &nb, st()));
        CC_CUDA(M2Launch<T>::phi_to_field(sphi, nx, ny, phi, P, active(), st()));
        count(3);
        return CC_OK;
    }

    DtSpec dtspec(bool clamp) const {
        const double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
        DtSpec d;
        d.cfl = p.cfl; d.hmin = vmin(dx, dy); d.eta = 0.0; d.t_end = p.t_end; d.clamp_to_end = clamp ? 1 : 0;
        d.seed = 1e-30; d.end_eps = 1e-14; d.check = 1; d.cap = 0;   // EH:395, 697, 699-702
        return d;
    }

    int compute_dt(double* dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        CC_CUDA(EHLaunch<T>::speeds(c, U, spd_part, rho_part, st()));
        CC_CUDA(launch_dt_finalize(spd_part, dtspec(false), dt_dev(), t_dev(), active(), st()));
        count(2);
        CC_CUDA(cudaMemcpyAsync(dt, dt_dev(), sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int gravity(double* gx, double* gy) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        const int nx = p.Nx, ny = p.Ny;
        int one = 1;
        CC_CUDA(cudaMemcpyAsync(iflags, &one, sizeof(int), cudaMemcpyHostToDevice, st()));
        if (p.gravity_on) {
            if (!radial()) {
                CC_CUDA(EHLaunch<T>::rho_sum(c, U.rho, rho_part, st()));
                count(1);
            }
            if (int r = solve(U.rho)) return r;
        }
        if (!g2[0]) {
            CC_CUDA(cudaMalloc(&g2[0], sizeof(T) * plane));
            CC_CUDA(cudaMalloc(&g2[1], sizeof(T) * plane));
        }
        if (radial()) {
            // g2 holds the enclosed-mass gravity from solve()
        } else if (p.gravity_on) {
            CC_CUDA(M2Launch<T>::gravity_from_phi(phi, nx, ny, P, c.pax, c.pay, c.two_dx, c.two_dy, g2[0], g2[1], st()));
            count(1);
        } else {
            CC_CUDA(cudaMemsetAsync(g2[0], 0, sizeof(T) * plane, st()));
            CC_CUDA(cudaMemsetAsync(g2[1], 0, sizeof(T) * plane, st()));
        }
        double* dst[2] = {gx, gy};
        for (int k = 0; k < 2; k++) {
            if (!dst[k]) continue;
            CC_CUDA(M2Launch<T>::pack_out(g2[k], staging, nx, ny, P, st()));
            count(1);
            CC_CUDA(cudaMemcpyAsync(dst[k], staging, sizeof(double) * (size_t)nx * ny, cudaMemcpyDeviceToHost, st()));
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return check_flags();
    }

    int check_flags() {
        int fl[4];
        CC_CUDA(cudaMemcpy(fl, iflags, sizeof(fl), cudaMemcpyDeviceToHost));
        if (fl[1]) return fail(h, CC_ERR_CUDA, "SOR grid barrier timed out");
        if (fl[3]) return fail(h, CC_ERR_NONFINITE, "dt not finite or not positive (the reference aborts here)");
        return CC_OK;
    }

    // rk2_step (EH:529-550) with dt in dt_dev; the RHS solves Poisson itself (EH:411)
    int step_body() {
        if (p.gravity_on) {
            if (!radial()) {   // the SOR's density mean
                CC_CUDA(EHLaunch<T>::rho_sum(c, U.rho, rho_part, st()));
                count(1);
            }
            if (int r = solve(U.rho)) return r;
        }
        CC_CUDA(EHLaunch<T>::stage(c, U, U, U1, false, phi, gxa(), gya(), dt_dev(), active(), st()));
        count(1);
        if (p.gravity_on) {
            if (!radial()) {
                CC_CUDA(EHLaunch<T>::rho_sum(c, U1.rho, rho_part, st()));
                count(1);
            }
            if (int r = solve(U1.rho)) return r;
        }
        CC_CUDA(EHLaunch<T>::stage(c, U, U1, U, true, phi, gxa(), gya(), dt_dev(), active(), st()));
        count(1);
        h->perf.steps += 1;
        return CC_OK;
    }

    int rk2_step(double dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        int one = 1;
        CC_CUDA(cudaMemcpyAsync(iflags, &one, sizeof(int), cudaMemcpyHostToDevice, st()));
        CC_CUDA(launch_set_scalar(dt_dev(), dt, st()));
        count(1);
        if (int r = step_body()) return r;
        CC_CUDA(cudaStreamSynchronize(st()));
        return check_flags();
    }

    int device_step() {
        CC_CUDA(EHLaunch<T>::speeds(c, U, spd_part, rho_part, st()));
        CC_CUDA(launch_dt_finalize(spd_part, dtspec(true), dt_dev(), t_dev(), active(), st()));
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
        const bool graphable = !p.gravity_on && !h->profiling;
        if (graphable && nsteps >= 1) {
            if (!graph1 || graph_stream != st()) {
                if (graph1) { cudaGraphExecDestroy(graph1); graph1 = nullptr; }
                const cc_perf before = h->perf;
                cudaGraph_t g = nullptr;
                CC_CUDA(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
                int rr = device_step();
                cudaError_t e = cudaStreamEndCapture(st(), &g);
                graph_delta.kernel_launches = h->perf.kernel_launches - before.kernel_launches;
                graph_delta.steps = h->perf.steps - before.steps;
                h->perf = before;
                if (rr) { if (g) cudaGraphDestroy(g); return rr; }
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
                e = cudaGraphInstantiate(&graph1, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
                graph_stream = st();
            }
            for (int k = 0; k < nsteps; k++) {
                CC_CUDA(cudaGraphLaunch(graph1, st()));
                h->perf.kernel_launches += graph_delta.kernel_launches;
                h->perf.steps += graph_delta.steps;
            }
        } else {
            for (int k = 0; k < nsteps; k++)
                if (int r = device_step()) return r;
        }
        if (t) CC_CUDA(cudaMemcpyAsync(t, t_dev(), sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return check_flags();
    }

    int derived(double* const* out) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        const size_t n = (size_t)p.Nx * p.Ny;
        if (!derived_dev) CC_CUDA(cudaMalloc(&derived_dev, sizeof(double) * n * 3));
        CC_CUDA(EHLaunch<T>::derived(c, U, derived_dev, st()));
        count(1);
        for (int k = 0; k < 3; k++)
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

    const cc_euler2d_params& params() const override { return p; }

    int diagnostics(cc_diag* d) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        CC_CUDA(EHLaunch<T>::diag(c, U, diag_part, st()));
        count(1);
        std::vector<double> part(RED_BLOCKS * 5);
        CC_CUDA(cudaMemcpyAsync(part.data(), diag_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st()));
        double sc[4];
        CC_CUDA(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st()));
        long long steps = 0;
        CC_CUDA(cudaMemcpyAsync(&steps, steps_dev, sizeof(steps), cudaMemcpyDeviceToHost, st()));
        int fl[4];
        CC_CUDA(cudaMemcpyAsync(fl, iflags, sizeof(fl), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        double s[4] = {0, 0, 0, 0}, nonf = 0.0;
        for (int m = 0; m < 4; m++)
            for (int b = 0; b < RED_BLOCKS; b++) s[m] += part[m * RED_BLOCKS + b];
        for (int b = 0; b < RED_BLOCKS; b++) nonf = std::fmax(nonf, part[4 * RED_BLOCKS + b]);
        const double dV = ((p.x1 - p.x0) / p.Nx) * ((p.y1 - p.y0) / p.Ny);
        std::memset(d, 0, sizeof(*d));
        d->mass = s[0] * dV; d->mom_x = s[1] * dV; d->mom_y = s[2] * dV; d->energy = s[3] * dV;
        d->t = sc[1]; d->dt_last = sc[0]; d->steps = steps;
        d->poisson_iters = fl[2]; d->poisson_residual = sc[2];
        d->nonfinite = nonf > 0.0 ? 1 : 0;
        return CC_OK;
    }
};

struct Euler2dHandle : cc_handle {
    std::unique_ptr<Euler2dBase> impl;
};

Euler2dBase* eh(cc_handle* h) {
    if (!h || h->kind != KIND_EULER2D) return nullptr;
    return static_cast<Euler2dHandle*>(h)->impl.get();
}

}  // namespace

extern "C" {

void cc_euler2d_params_default(cc_euler2d_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma = 1.2; p->cfl = 0.45;
    p->x0 = 0.0; p->x1 = 1.0; p->y0 = 0.0; p->y1 = 1.0;
    p->Nx = 50; p->Ny = 50;
    p->t_end = 5.0; p->dt_store = 1e-3;
    p->floor_rho = 1e-12; p->floor_P = 1e-12;
    p->periodic_x = 1; p->periodic_y = 1;
    p->gravity_on = 1; p->sor_max_iter = 50000;
    p->G = 1.0; p->softening = 1e-4;
    p->sor_tol = 1e-10; p->sor_omega = 1.7;
    p->poisson_kind = CC_POISSON_SOR; p->precision = CC_FP64;
    p->Nr_bins = 512; p->xc = 0.5; p->yc = 0.5;
}

int cc_euler2d_create(const cc_euler2d_params* p, cc_handle** out) {
    if (!p || !out) return CC_ERR_ARG;
    *out = nullptr;
    if (p->Nx < 2 || p->Ny < 2 || !(p->x1 > p->x0) || !(p->y1 > p->y0)) return CC_ERR_ARG;
    if (p->precision != CC_FP64 && p->precision != CC_FP32) return CC_ERR_ARG;
    auto h = std::make_unique<Euler2dHandle>();
    h->kind = KIND_EULER2D;
    if (cudaGetDevice(&h->device) != cudaSuccess) return CC_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return CC_ERR_CUDA;
    h->stream = h->own;
    if (p->precision == CC_FP64) h->impl = std::make_unique<Euler2d<double>>(h.get(), *p);
    else h->impl = std::make_unique<Euler2d<float>>(h.get(), *p);
    int r = h->impl->init();
    *out = h.release();
    return r;
}

int cc_euler2d_upload(cc_handle* h, const double* rho, const double* mx, const double* my, const double* E) {
    Euler2dBase* m = eh(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const double* f[4] = {rho, mx, my, E};
    return m->upload(f);
}

int cc_euler2d_download(cc_handle* h, double* rho, double* mx, double* my, double* E) {
    Euler2dBase* m = eh(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    double* f[4] = {rho, mx, my, E};
    return m->download(f);
}

int cc_euler2d_compute_dt(cc_handle* h, double* dt) {
    Euler2dBase* m = eh(h);
    if (!m || !dt) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->compute_dt(dt);
}

int cc_euler2d_compute_gravity(cc_handle* h, double* gx, double* gy) {
    Euler2dBase* m = eh(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->gravity(gx, gy);
}

int cc_euler2d_rk2_step(cc_handle* h, double dt) {
    Euler2dBase* m = eh(h);
    if (!m) return CC_ERR_ARG;
    if (!std::isfinite(dt) || dt <= 0.0) return fail(h, CC_ERR_NONFINITE, "dt not finite or not positive");
    if (int r = set_dev(h)) return r;
    return m->rk2_step(dt);
}

int cc_euler2d_advance(cc_handle* h, int nsteps, double* t) {
    Euler2dBase* m = eh(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->advance(nsteps, t);
}

int cc_euler2d_diagnostics(cc_handle* h, cc_diag* d) {
    Euler2dBase* m = eh(h);
    if (!m || !d) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->diagnostics(d);
}

int cc_euler2d_derived(cc_handle* h, double* const* out) {
    Euler2dBase* m = eh(h);
    if (!m || !out) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->derived(out);
}

// restart files (checkpoint.h): state {rho, mx, my, E} and the clock
int cc_euler2d_checkpoint_save(cc_handle* h, const char* path) {
    Euler2dBase* m = eh(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_euler2d_params& p = m->params();
    const size_t n = (size_t)p.Nx * p.Ny;
    std::vector<std::vector<double>> f(4, std::vector<double>(n));
    double* fp[4] = {f[0].data(), f[1].data(), f[2].data(), f[3].data()};
    if (int r = m->download(fp)) return r;
    CkMeta meta;
    meta.precision = (uint32_t)p.precision;
    meta.n[0] = p.Nx; meta.n[1] = p.Ny;
    if (int r = m->get_clock(&meta.t, &meta.steps)) return r;
    std::string err;
    if (int r = ck3_save(path, "CCEH2CK1", meta, &p, sizeof(p), f, err)) return fail(h, r, err);
    return CC_OK;
}

int cc_euler2d_checkpoint_load(cc_handle* h, const char* path) {
    Euler2dBase* m = eh(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_euler2d_params& p = m->params();
    CkMeta meta;
    cc_euler2d_params q;
    std::vector<std::vector<double>> f;
    std::string err;
    auto sizes = [](const int32_t* n) { return std::vector<size_t>(4, (size_t)n[0] * n[1]); };
    if (int r = ck3_load(path, "CCEH2CK1", meta, &q, sizeof(q), sizes, f, err)) return fail(h, r, err);
    if (meta.n[0] != p.Nx || meta.n[1] != p.Ny || (int)meta.precision != p.precision || q.x0 != p.x0 ||
        q.x1 != p.x1 || q.y0 != p.y0 || q.y1 != p.y1 || q.periodic_x != p.periodic_x || q.periodic_y != p.periodic_y)
        return fail(h, CC_ERR_ARG, "checkpoint grid, domain, boundaries or precision differ from the handle's");
    const double* fp[4] = {f[0].data(), f[1].data(), f[2].data(), f[3].data()};
    if (int r = m->upload(fp)) return r;
    return m->set_clock(meta.t, meta.steps);
}

}  // extern "C"
