// Host side of the batched 2D MHD ensemble: the Batch<T> solver object
// (device pool, work-lists, direct-Poisson set-up, step orchestration), shared
// by the ensemble C ABI (capi_batch.cu) and the discrete adjoint
// (capi_adjoint.cu).  Internal linkage: each including translation unit gets
// its own copy.
#pragma once
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/cc_batch.h"
#include "batch_launch.h"
#include "handle.h"
#include "mhd2d_launch.h"

namespace {

using namespace ccb;


constexpr int KIND_BATCH = 4;

// Orthonormal eigenbasis of the x second difference and its eigenvalues:
// DCT-II for the clamp rule, discrete Hartley for the periodic rule (the CPU
// oracle builds the same values with the same expressions).
void x_basis(int n, bool periodic, double d, std::vector<double>& tx, std::vector<double>& lam) {
    tx.assign((size_t)n * n, 0.0);
    lam.assign(n, 0.0);
    for (int k = 0; k < n; k++) {
        double sn;
        if (periodic) {
            const double sc = 1.0 / std::sqrt((double)n);
            for (int i = 0; i < n; i++) {
                const double arg = 2.0 * M_PI * (double)(((long long)k * i) % n) / (double)n;
                tx[(size_t)k * n + i] = (std::cos(arg) + std::sin(arg)) * sc;
            }
            sn = std::sin(M_PI * (double)k / (double)n);
        } else {
            const double sc = std::sqrt((k == 0 ? 1.0 : 2.0) / (double)n);
            for (int i = 0; i < n; i++) {
                const double arg = M_PI * (double)((long long)k * (2 * i + 1)) / (double)(2 * n);
                tx[(size_t)k * n + i] = sc * std::cos(arg);
            }
            sn = std::sin(M_PI * (double)k / (double)(2 * n));
        }
        lam[k] = -4.0 * sn * sn / (d * d);
    }
}

// Factors of the y systems (Dyy + lam_k) u = r of every x wavenumber k >= 1
// of a grid, stored [j*nx + k]: m_j = b_j - a cp_{j-1} (fma), inv_j = 1/m_j,
// cp_j = a inv_j, clamp end rows b = lam - a; periodic y: Sherman-Morrison
// with gamma = -b (rows 0 and n-1 of T' modified), z = T'^-1 (gamma, 0.., a)
// and fden = 1 / (1 + v.z).  The CPU oracle sets up the same values the same way.
void y_factors(int nx, int ny, bool py, double a, const std::vector<double>& lam, std::vector<double>& cp,
               std::vector<double>& inv, std::vector<double>& z, std::vector<double>& fden) {
    cp.assign((size_t)nx * ny, 0.0);
    inv.assign((size_t)nx * ny, 0.0);
    z.assign(py ? (size_t)nx * ny : 0, 0.0);
    fden.assign(nx, 0.0);
    for (int k = 1; k < nx; k++) {
        const double lk = lam[k];
        const double b = std::fma(-2.0, a, lk);
        const double gam = -b;
        const double bE = py ? b - gam : lk - a;
        const double bL = py ? b - a * a / gam : lk - a;
        double cprev = 0.0;
        for (int j = 0; j < ny; j++) {
            const double bj = (j == 0) ? bE : (j == ny - 1 ? bL : b);
            const double m = (j == 0) ? bj : std::fma(-a, cprev, bj);
            const double iv = 1.0 / m;
            inv[(size_t)j * nx + k] = iv;
            cprev = a * iv;
            cp[(size_t)j * nx + k] = cprev;
        }
        if (py) {
            for (int j = 0; j < ny; j++) {
                const double zr = (j == 0) ? gam : (j == ny - 1 ? a : 0.0);
                const double iv = inv[(size_t)j * nx + k];
                z[(size_t)j * nx + k] = (j == 0) ? zr * iv : std::fma(-a, z[(size_t)(j - 1) * nx + k], zr) * iv;
            }
            for (int j = ny - 2; j >= 0; j--)
                z[(size_t)j * nx + k] = std::fma(-cp[(size_t)j * nx + k], z[(size_t)(j + 1) * nx + k], z[(size_t)j * nx + k]);
            fden[k] = 1.0 / (1.0 + std::fma(a / gam, z[(size_t)(ny - 1) * nx + k], z[k]));
        }
    }
}

struct BatchBase {
    virtual ~BatchBase() {}
    virtual int init() = 0;
    virtual int upload(int inst, const double* const* f) = 0;
    virtual int download(int inst, double* const* f) = 0;
    virtual int compute_dt(double* dt) = 0;
    virtual int advance(int nsteps, double* t) = 0;
    virtual int diagnostics(int inst, cc_diag* d) = 0;
    virtual int times(double* t) = 0;
    virtual int autotune(int reps, int* shape, double* ms) = 0;
    virtual int set_shape(int shape) = 0;
    virtual int info(cc_batch_info* out) = 0;
};

template <class T> struct Batch : BatchBase {
    cc_handle* h;
    std::vector<cc_mhd2d_params> p;
    int n;
    std::vector<BatchInst<T>> hinst;
    std::vector<BatchRed> hred;
    std::vector<int> pitch;
    BatchInst<T>* dinst = nullptr;
    BatchRed* dred = nullptr;
    std::vector<void*> allocs;
    size_t bytes = 0;
    // work-lists
    // stage candidates: tile shape k = c % NS, launched persistent (c < NS:
    // one CTA per resident slot, each walking a contiguous run of the
    // work-list) or flat (c >= NS: one CTA per tile, scheduled by hardware)
    std::vector<int2*> swork;        // per stage shape
    std::vector<int> nswork;
    std::vector<int> sgrid;          // CTAs per candidate
    int2* rwork = nullptr; int nrwork = 0;
    int2* gwork = nullptr; int ngwork = 0; int gtile = 64;
    int2* tcwork = nullptr; int ntcwork = 0;   // FP32 instances with 16-byte rows: tcgen05 transforms
    int* tcerr = nullptr;            // timed-out waits of the tensor-core transforms (bit 0; bit 1: the final
                                     // wait for the MMAs gave up too)
    bool tc_fatal = false;           // bit 1 was seen: MMAs may have outlived their TMEM, no further work
    int2* ywork = nullptr; int nywork = 0;
    // per-instance device scalars and partials
    double* spd_part = nullptr;
    double* rho_part = nullptr;
    double* dt = nullptr;
    double* tclk = nullptr;
    double* rho_mean = nullptr;
    int* active = nullptr;
    long long* steps = nullptr;
    double* diag_part = nullptr;
    double* staging = nullptr;
    size_t staging_elems = 0;
    bool any_grav = false;
    int shape = 0;
    int cur = 0;
    std::vector<char> loaded;
    bool partials_valid = false;
    cudaGraphExec_t graph3 = nullptr;
    cudaStream_t graph_stream = nullptr;
    int graph_cur = -1;
    int graph_shape = -1;
    cc_perf graph_delta{};

    Batch(cc_handle* hh, const cc_mhd2d_params* pp, int nn) : h(hh), p(pp, pp + nn), n(nn) {}
    cc_handle* this_handle() { return h; }
    cudaStream_t st() const { return h->stream; }

    ~Batch() override {
        if (graph3) cudaGraphExecDestroy(graph3);
        for (void* q : allocs) cudaFree(q);
    }

    template <class U> int dalloc(U** ptr, size_t count) {
        void* q = nullptr;
        CC_CUDA(cudaMalloc(&q, sizeof(U) * (count ? count : 1)));
        allocs.push_back(q);
        bytes += sizeof(U) * (count ? count : 1);
        *ptr = reinterpret_cast<U*>(q);
        return CC_OK;
    }
    template <class U> int upload_vec(U** ptr, const std::vector<U>& v) {
        if (int r = dalloc(ptr, v.size())) return r;
        if (!v.empty()) CC_CUDA(cudaMemcpyAsync(*ptr, v.data(), sizeof(U) * v.size(), cudaMemcpyHostToDevice, st()));
        return CC_OK;
    }

    int init() override {
        CC_CUDA(BatchLaunch<T>::prepare());
        CC_CUDA(DPoissonLaunch<T>::prepare());
        hinst.resize(n);
        hred.resize(n);
        pitch.resize(n);
        loaded.assign(n, 0);
        // ---- state pool: 3 x 8 planes + phi per instance ----
        std::vector<size_t> off(n);
        size_t total = 0;
        for (int i = 0; i < n; i++) {
            const cc_mhd2d_params& q = p[i];
            pitch[i] = ((q.Nx + 1 + 31) / 32) * 32;
            off[i] = total;
            total += (size_t)pitch[i] * (q.Ny + 1) * 25;
            staging_elems = std::max(staging_elems, (size_t)(q.Nx + 1) * (q.Ny + 1));
            if (q.gravity_on) any_grav = true;
        }
        T* pool = nullptr;
        if (int r = dalloc(&pool, total)) return r;
        CC_CUDA(cudaMemsetAsync(pool, 0, sizeof(T) * total, st()));
        // ---- direct Poisson: x bases per (nx, periodic, dx), y factors per grid shape ----
        // (built in FP64, stored in the state precision T)
        std::map<std::tuple<int, int, double>, std::tuple<T*, T*, T*>> bases;
        std::map<std::tuple<int, int, double, int, int, double>, std::tuple<T*, T*, T*, T*>> yfac;
        auto to_t = [](const std::vector<double>& v) { return std::vector<T>(v.begin(), v.end()); };
        for (int i = 0; i < n; i++) {
            const cc_mhd2d_params& q = p[i];
            const int nx = q.Nx, ny = q.Ny, P = pitch[i];
            const double dx = (q.x1 - q.x0) / nx, dy = (q.y1 - q.y0) / ny;
            BatchInst<T>& I = hinst[i];
            std::memset(&I, 0, sizeof(I));
            M2Const<T>& c = I.c;
            c.gamma = (T)q.gamma;
            c.gm1 = (T)q.gamma - (T)1.0;
            c.floor_rho = (T)q.floor_rho;
            c.floor_P = (T)q.floor_P;
            c.eta = (T)q.eta;
            c.dx = (T)dx; c.dy = (T)dy;
            c.inv_dx = (T)(1.0 / dx); c.inv_dy = (T)(1.0 / dy);
            c.idx2 = (T)(1.0 / (dx * dx)); c.idy2 = (T)(1.0 / (dy * dy));
            c.two_dx = (T)(2.0 * dx); c.two_dy = (T)(2.0 * dy);
            c.nx = nx; c.ny = ny; c.pitch = P;
            c.ax = AxisMap{nx, q.periodic_x ? 1 : 0};
            c.ay = AxisMap{ny, q.periodic_y ? 1 : 0};
            c.gravity_on = q.gravity_on ? 1 : 0;
            c.resistive = (q.eta > 0.0) ? 1 : 0;
            const size_t plane = (size_t)P * (ny + 1);
            T* base = pool + off[i];
            for (int b = 0; b < 3; b++) {
                T* s = base + (size_t)b * 8 * plane;
                I.buf[b] = Fields<T>{s, s + plane, s + 2 * plane, s + 3 * plane,
                                     s + 4 * plane, s + 5 * plane, s + 6 * plane, s + 7 * plane};
            }
            I.phi = base + 24 * plane;
            I.fourpiG = 4.0 * M_PI * q.G;
            I.ay = 1.0 / (dy * dy);
            I.dy2 = dy * dy;
            if (q.gravity_on) {
                auto key = std::make_tuple(nx, q.periodic_x ? 1 : 0, dx);
                auto it = bases.find(key);
                if (it == bases.end()) {
                    std::vector<double> tx, lam;
                    x_basis(nx, q.periodic_x != 0, dx, tx, lam);
                    std::vector<double> txt((size_t)nx * nx);
                    for (int a = 0; a < nx; a++)
                        for (int b = 0; b < nx; b++) txt[(size_t)b * nx + a] = tx[(size_t)a * nx + b];
                    T *d_tx, *d_txt, *d_lam;
                    if (int r = upload_vec(&d_tx, to_t(tx))) return r;
                    if (int r = upload_vec(&d_txt, to_t(txt))) return r;
                    if (int r = upload_vec(&d_lam, to_t(lam))) return r;
                    it = bases.emplace(key, std::make_tuple(d_tx, d_txt, d_lam)).first;
                }
                I.tx = std::get<0>(it->second);
                I.txt = std::get<1>(it->second);
                I.lamx = std::get<2>(it->second);
                auto ykey = std::make_tuple(nx, q.periodic_x ? 1 : 0, dx, ny, q.periodic_y ? 1 : 0, dy);
                auto yt = yfac.find(ykey);
                if (yt == yfac.end()) {
                    std::vector<double> tx, lam, cp, inv, z, fden;
                    x_basis(nx, q.periodic_x != 0, dx, tx, lam);
                    y_factors(nx, ny, q.periodic_y != 0, 1.0 / (dy * dy), lam, cp, inv, z, fden);
                    T *d_cp, *d_inv, *d_z = nullptr, *d_fden;
                    if (int r = upload_vec(&d_cp, to_t(cp))) return r;
                    if (int r = upload_vec(&d_inv, to_t(inv))) return r;
                    if (q.periodic_y)
                        if (int r = upload_vec(&d_z, to_t(z))) return r;
                    if (int r = upload_vec(&d_fden, to_t(fden))) return r;
                    yt = yfac.emplace(ykey, std::make_tuple(d_cp, d_inv, d_z, d_fden)).first;
                }
                I.ycp = std::get<0>(yt->second);
                I.yinv = std::get<1>(yt->second);
                I.yz = std::get<2>(yt->second);
                I.yfden = std::get<3>(yt->second);
                if (int r = dalloc(&I.ah, (size_t)nx * ny)) return r;
            }
            BatchRed& R = hred[i];
            R.ncell = (double)nx * (double)ny;
            const double hmin = std::fmin(dx, dy);
            R.dts.cfl = q.cfl; R.dts.hmin = hmin; R.dts.eta = q.eta; R.dts.t_end = q.t_end;
            R.dts.clamp_to_end = 1; R.dts.seed = 1e-14; R.dts.end_eps = 0.0; R.dts.check = 0; R.dts.cap = 1;
        }
        // ---- work-lists ----
        std::vector<int2> rw, gw, gw32, gw128, yw;
        for (int i = 0; i < n; i++) {
            const int nx = p[i].Nx, ny = p[i].Ny;
            hred[i].base = (int)rw.size();
            for (int ty = 0; ty < (ny + RTY - 1) / RTY; ty++)
                for (int tx = 0; tx < (nx + RTX - 1) / RTX; tx++) rw.push_back(make_int2(i, (ty << 16) | tx));
            hred[i].count = (int)rw.size() - hred[i].base;
            if (p[i].gravity_on) {
                // per instance (so that its result does not depend on the batch):
                // FP32 with 16-byte rows on the tensor cores, else CUDA cores
                if (sizeof(T) == 4 && nx % 4 == 0) {
                    for (int tm = 0; tm < (ny + 127) / 128; tm++)
                        for (int tn = 0; tn < (nx + 127) / 128; tn++) gw128.push_back(make_int2(i, (tm << 16) | tn));
                } else {
                    for (int tm = 0; tm < (ny + 63) / 64; tm++)
                        for (int tn = 0; tn < (nx + 63) / 64; tn++) gw.push_back(make_int2(i, (tm << 16) | tn));
                    for (int tm = 0; tm < (ny + 31) / 32; tm++)
                        for (int tn = 0; tn < (nx + 31) / 32; tn++) gw32.push_back(make_int2(i, (tm << 16) | tn));
                }
                // item -1: the singular x wavenumber 0 on its own; items cb >= 0:
                // wavenumbers 1 + 32 cb + lane
                yw.push_back(make_int2(i, -1));
                for (int cb = 0; cb < (nx - 1 + 31) / 32; cb++) yw.push_back(make_int2(i, cb));
            }
        }
        // CUDA-core GEMMs on 64 x 64 tiles unless they would leave most SMs
        // idle (small batches); same per-output k order, same bits
        if (gw.size() < 296) { gw.swap(gw32); gtile = 32; }
        ntcwork = (int)gw128.size();
        if (int r = upload_vec(&tcwork, gw128)) return r;
        if (int r = dalloc(&tcerr, 1)) return r;
        CC_CUDA(cudaMemsetAsync(tcerr, 0, sizeof(int), st()));
        nrwork = (int)rw.size(); ngwork = (int)gw.size(); nywork = (int)yw.size();
        if (int r = upload_vec(&rwork, rw)) return r;
        if (int r = upload_vec(&gwork, gw)) return r;
        if (int r = upload_vec(&ywork, yw)) return r;
        int dev = 0, nsm = 0;
        CC_CUDA(cudaGetDevice(&dev));
        CC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const int NS = BatchLaunch<T>::n_shapes();
        swork.assign(NS, nullptr);
        nswork.assign(NS, 0);
        sgrid.assign(2 * NS, 1);
        for (int k = 0; k < NS; k++) {
            const TileShape sh = BatchLaunch<T>::shape(k);
            std::vector<int2> sw;
            for (int i = 0; i < n; i++) {
                const int nx = p[i].Nx, ny = p[i].Ny;
                for (int ty = 0; ty < (ny + sh.ty - 1) / sh.ty; ty++)
                    for (int tx = 0; tx < (nx + sh.tx - 1) / sh.tx; tx++) sw.push_back(make_int2(i, (ty << 16) | tx));
            }
            nswork[k] = (int)sw.size();
            if (int r = upload_vec(&swork[k], sw)) return r;
            int per_sm = 0;
            CC_CUDA(BatchLaunch<T>::resident(k, &per_sm));
            if (per_sm < 1) per_sm = 1;
            sgrid[k] = std::max(1, std::min(nswork[k], per_sm * nsm));
            sgrid[NS + k] = std::max(1, nswork[k]);
        }
        if (int r = upload_vec(&dinst, hinst)) return r;
        if (int r = upload_vec(&dred, hred)) return r;
        if (int r = dalloc(&spd_part, nrwork)) return r;
        if (int r = dalloc(&rho_part, nrwork)) return r;
        if (int r = dalloc(&dt, n)) return r;
        if (int r = dalloc(&tclk, n)) return r;
        if (int r = dalloc(&rho_mean, n)) return r;
        if (int r = dalloc(&active, n)) return r;
        if (int r = dalloc(&steps, n)) return r;
        if (int r = dalloc(&diag_part, (size_t)RED_BLOCKS * 7)) return r;
        if (int r = dalloc(&staging, staging_elems)) return r;
        CC_CUDA(cudaMemsetAsync(dt, 0, sizeof(double) * n, st()));
        CC_CUDA(cudaMemsetAsync(tclk, 0, sizeof(double) * n, st()));
        CC_CUDA(cudaMemsetAsync(rho_mean, 0, sizeof(double) * n, st()));
        CC_CUDA(cudaMemsetAsync(steps, 0, sizeof(long long) * n, st()));
        CC_CUDA(launch_batch_set_active(n, active, 1, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    void invalidate_graph() {
        if (graph3) { cudaGraphExecDestroy(graph3); graph3 = nullptr; }
    }

    void layout(int i, int* w, int* hh) const {
        const int nx = p[i].Nx, ny = p[i].Ny;
        const int ww[8] = {nx, nx, nx, nx, nx, nx, nx + 1, nx};
        const int hv[8] = {ny, ny, ny, ny, ny, ny, ny, ny + 1};
        for (int k = 0; k < 8; k++) { w[k] = ww[k]; hh[k] = hv[k]; }
    }

    int upload(int i, const double* const* f) override {
        if (tc_fatal) return fail(h, CC_ERR_CUDA, "handle unusable: an earlier tensor-core transform gave up on its MMAs");
        if (i < 0 || i >= n || !f) return fail(h, CC_ERR_ARG, "bad instance index or null state");
        int w[8], hh[8];
        layout(i, w, hh);
        const Fields<T>& B = hinst[i].buf[cur];
        T* dst[8] = {B.rho, B.mx, B.my, B.mz, B.E, B.Bz, B.bx, B.by};
        for (int k = 0; k < 8; k++) {
            if (!f[k]) return fail(h, CC_ERR_ARG, "null state array");
            CC_CUDA(cudaMemcpyAsync(staging, f[k], sizeof(double) * (size_t)w[k] * hh[k], cudaMemcpyHostToDevice, st()));
            CC_CUDA(M2Launch<T>::pack_in(staging, dst[k], w[k], hh[k], pitch[i], st()));
            h->perf.kernel_launches += 1;
        }
        loaded[i] = 1;
        partials_valid = false;
        return CC_OK;
    }

    bool all_loaded() const {
        for (char c : loaded)
            if (!c) return false;
        return true;
    }

    int download(int i, double* const* f) override {
        if (i < 0 || i >= n || !f) return fail(h, CC_ERR_ARG, "bad instance index or null state");
        if (!loaded[i]) return fail(h, CC_ERR_STATE, "instance has no uploaded state");
        int w[8], hh[8];
        layout(i, w, hh);
        const Fields<T>& B = hinst[i].buf[cur];
        const T* src[8] = {B.rho, B.mx, B.my, B.mz, B.E, B.Bz, B.bx, B.by};
        for (int k = 0; k < 8; k++) {
            if (!f[k]) continue;
            CC_CUDA(M2Launch<T>::pack_out(src[k], staging, w[k], hh[k], pitch[i], st()));
            CC_CUDA(cudaMemcpyAsync(f[k], staging, sizeof(double) * (size_t)w[k] * hh[k], cudaMemcpyDeviceToHost, st()));
            h->perf.kernel_launches += 1;
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    void count(int k) { h->perf.kernel_launches += k; }

    int ensure_partials() {
        if (partials_valid) return CC_OK;
        CC_CUDA(BatchLaunch<T>::speeds(dinst, rwork, nrwork, cur, spd_part, rho_part, st()));
        count(1);
        partials_valid = true;
        return CC_OK;
    }

    int compute_dt(double* out) override {
        if (tc_fatal) return fail(h, CC_ERR_CUDA, "handle unusable: an earlier tensor-core transform gave up on its MMAs");
        if (!all_loaded()) return fail(h, CC_ERR_STATE, "not every instance has an uploaded state");
        if (int r = ensure_partials()) return r;
        CC_CUDA(launch_batch_finalize(dred, n, spd_part, rho_part, BF_DT, dt, tclk, active, rho_mean, st()));
        count(1);
        CC_CUDA(cudaMemcpyAsync(out, dt, sizeof(double) * n, cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    // density means from rho_part, then the direct solve on buffer src
    int poisson(int src) {
        CC_CUDA(launch_batch_finalize(dred, n, spd_part, rho_part, BF_MEAN, dt, tclk, active, rho_mean, st()));
        CC_CUDA(DPoissonLaunch<T>::solve(dinst, gwork, ngwork, gtile, tcwork, ntcwork, ywork, nywork, src, rho_mean,
                                         active, tcerr, st()));
        count(4);
        h->perf.poisson_solves += 1;
        return CC_OK;
    }

    int stage(int src, int dst_, bool defer) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (h->profiling) {
            CC_CUDA(cudaEventCreate(&e0));
            CC_CUDA(cudaEventCreate(&e1));
            CC_CUDA(cudaEventRecord(e0, st()));
        }
        const int k = shape % BatchLaunch<T>::n_shapes();
        CC_CUDA(BatchLaunch<T>::stage(k, sgrid[shape], dinst, swork[k], nswork[k], src, dst_, defer, any_grav, dt,
                                      active, st()));
        count(1);
        if (h->profiling) {
            CC_CUDA(cudaEventRecord(e1, st()));
            h->timed.emplace_back(e0, e1);
        }
        return CC_OK;
    }

    int device_step() {
        if (int r = ensure_partials()) return r;
        const int a = cur, b = (cur + 1) % 3, d = (cur + 2) % 3;
        if (any_grav)
            if (int r = poisson(a)) return r;
        CC_CUDA(launch_batch_finalize(dred, n, spd_part, rho_part, BF_DT | BF_CLAMP, dt, tclk, active, rho_mean, st()));
        count(1);
        if (int r = stage(a, b, false)) return r;
        if (any_grav) {
            CC_CUDA(BatchLaunch<T>::rho_sum(dinst, rwork, nrwork, b, active, rho_part, st()));
            count(1);
            if (int r = poisson(b)) return r;
        }
        if (int r = stage(b, d, true)) return r;
        CC_CUDA(BatchLaunch<T>::average(dinst, rwork, nrwork, a, d, b, dt, active, spd_part, rho_part, st()));
        CC_CUDA(launch_batch_clock(n, tclk, dt, active, steps, st()));
        count(2);
        h->perf.steps += 1;
        cur = b;
        partials_valid = true;
        return CC_OK;
    }

    int advance(int nsteps, double* t) override {
        if (tc_fatal) return fail(h, CC_ERR_CUDA, "handle unusable: an earlier tensor-core transform gave up on its MMAs");
        if (!all_loaded()) return fail(h, CC_ERR_STATE, "not every instance has an uploaded state");
        if (nsteps < 0) return fail(h, CC_ERR_ARG, "nsteps < 0");
        if (t) CC_CUDA(cudaMemcpyAsync(tclk, t, sizeof(double) * n, cudaMemcpyHostToDevice, st()));
        if (int r = ensure_partials()) return r;
        int done = 0;
        if (!h->profiling && nsteps >= 3) {
            if (!graph3 || graph_cur != cur || graph_stream != st() || graph_shape != shape) {
                invalidate_graph();
                const int start = cur;
                const cc_perf before = h->perf;
                cudaGraph_t g = nullptr;
                CC_CUDA(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
                int rr = CC_OK;
                for (int k = 0; k < 3 && rr == CC_OK; k++) rr = device_step();
                cudaError_t e = cudaStreamEndCapture(st(), &g);
                cur = start;
                graph_delta.kernel_launches = h->perf.kernel_launches - before.kernel_launches;
                graph_delta.poisson_solves = h->perf.poisson_solves - before.poisson_solves;
                graph_delta.steps = h->perf.steps - before.steps;
                h->perf = before;
                if (rr) { if (g) cudaGraphDestroy(g); return rr; }
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
                e = cudaGraphInstantiate(&graph3, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
                graph_cur = start;
                graph_stream = st();
                graph_shape = shape;
            }
            while (nsteps - done >= 3) {
                CC_CUDA(cudaGraphLaunch(graph3, st()));
                h->perf.kernel_launches += graph_delta.kernel_launches;
                h->perf.poisson_solves += graph_delta.poisson_solves;
                h->perf.steps += graph_delta.steps;
                done += 3;
            }
            partials_valid = true;
        }
        for (; done < nsteps; ++done)
            if (int r = device_step()) return r;
        if (t) CC_CUDA(cudaMemcpyAsync(t, tclk, sizeof(double) * n, cudaMemcpyDeviceToHost, st()));
        int terr = 0;
        CC_CUDA(cudaMemcpyAsync(&terr, tcerr, sizeof(int), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        if (terr & 2) tc_fatal = true;
        if (terr) return fail(h, CC_ERR_CUDA, "tensor-core Poisson transform: an mbarrier wait timed out");
        return CC_OK;
    }

    int times(double* t) override {
        CC_CUDA(cudaMemcpyAsync(t, tclk, sizeof(double) * n, cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int diagnostics(int i, cc_diag* d) override {
        if (i < 0 || i >= n || !d) return fail(h, CC_ERR_ARG, "bad instance index");
        if (!loaded[i]) return fail(h, CC_ERR_STATE, "instance has no uploaded state");
        const BatchInst<T>& I = hinst[i];
        CC_CUDA(M2Launch<T>::diag(I.c, I.buf[cur], diag_part, st()));
        count(1);
        std::vector<double> part(RED_BLOCKS * 7);
        CC_CUDA(cudaMemcpyAsync(part.data(), diag_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st()));
        double tt = 0.0, dd = 0.0;
        long long ss = 0;
        CC_CUDA(cudaMemcpyAsync(&tt, tclk + i, sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaMemcpyAsync(&dd, dt + i, sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaMemcpyAsync(&ss, steps + i, sizeof(long long), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        double s[5] = {0, 0, 0, 0, 0}, dmax = 0.0, nonf = 0.0;
        for (int m = 0; m < 5; m++)
            for (int b = 0; b < RED_BLOCKS; b++) s[m] += part[m * RED_BLOCKS + b];
        for (int b = 0; b < RED_BLOCKS; b++) {
            dmax = std::fmax(dmax, part[5 * RED_BLOCKS + b]);
            nonf = std::fmax(nonf, part[6 * RED_BLOCKS + b]);
        }
        const cc_mhd2d_params& q = p[i];
        const double dV = ((q.x1 - q.x0) / q.Nx) * ((q.y1 - q.y0) / q.Ny);
        std::memset(d, 0, sizeof(*d));
        d->mass = s[0] * dV; d->mom_x = s[1] * dV; d->mom_y = s[2] * dV; d->mom_z = s[3] * dV; d->energy = s[4] * dV;
        d->max_divB = dmax;
        d->t = tt;
        d->dt_last = dd;
        d->steps = ss;
        d->nonfinite = nonf > 0.0 ? 1 : 0;
        return CC_OK;
    }

    int autotune(int reps, int* out_shape, double* out_ms) override {
        if (tc_fatal) return fail(h, CC_ERR_CUDA, "handle unusable: an earlier tensor-core transform gave up on its MMAs");
        if (!all_loaded()) return fail(h, CC_ERR_STATE, "not every instance has an uploaded state");
        if (reps < 1) reps = 1;
        if (int r = ensure_partials()) return r;
        CC_CUDA(launch_batch_finalize(dred, n, spd_part, rho_part, BF_DT, dt, tclk, active, rho_mean, st()));
        const int b = (cur + 1) % 3;   // scratch buffer: the stage output is discarded
        cudaEvent_t e0, e1;
        CC_CUDA(cudaEventCreate(&e0));
        CC_CUDA(cudaEventCreate(&e1));
        int best = shape;
        double best_ms = 1e300;
        const int NS = BatchLaunch<T>::n_shapes();
        for (int c = 0; c < 2 * NS; c++) {
            const int k = c % NS;
            CC_CUDA(BatchLaunch<T>::stage(k, sgrid[c], dinst, swork[k], nswork[k], cur, b, false, any_grav, dt,
                                          active, st()));
            CC_CUDA(cudaEventRecord(e0, st()));
            for (int r = 0; r < reps; r++)
                CC_CUDA(BatchLaunch<T>::stage(k, sgrid[c], dinst, swork[k], nswork[k], cur, b, false, any_grav, dt,
                                              active, st()));
            CC_CUDA(cudaEventRecord(e1, st()));
            CC_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            CC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            count(reps + 1);
            const double per = (double)ms / reps;
            if (per < best_ms) { best_ms = per; best = c; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (best != shape) invalidate_graph();
        shape = best;
        if (out_shape) *out_shape = best;
        if (out_ms) *out_ms = best_ms;
        return CC_OK;
    }

    int set_shape(int k) override {
        if (k < 0 || k >= 2 * BatchLaunch<T>::n_shapes()) return fail(h, CC_ERR_ARG, "no such stage candidate");
        if (k != shape) invalidate_graph();
        shape = k;
        return CC_OK;
    }

    int info(cc_batch_info* o) override {
        std::memset(o, 0, sizeof(*o));
        o->n = n;
        o->precision = sizeof(T) == 8 ? CC_FP64 : CC_FP32;
        for (int i = 0; i < n; i++) o->cells += (long long)p[i].Nx * p[i].Ny;
        o->shape = shape;
        const int NS = BatchLaunch<T>::n_shapes();
        o->n_shapes = 2 * NS;
        const TileShape sh = BatchLaunch<T>::shape(shape % NS);
        o->tile_x = sh.tx; o->tile_y = sh.ty;
        o->stage_tiles = nswork[shape % NS];
        o->stage_ctas = sgrid[shape];
        o->reduce_tiles = nrwork;
        o->poisson_tiles = ngwork + ntcwork;
        o->poisson_tile = ntcwork > 0 ? (ngwork > 0 ? -128 : 128) : gtile;
        o->device_bytes = (int64_t)bytes;
        return CC_OK;
    }
};

}  // namespace
