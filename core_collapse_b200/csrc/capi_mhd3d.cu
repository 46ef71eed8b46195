// C ABI of the 3D MHD step (mhd3d_resistive_hlld_ct.cpp): handle, state
// transfer, compute_dt, rk2_step and the device-resident main-loop body.
//
// Per step (M3:1285-1291, 1034-1066): dt = finalize(CFL partials), clamped to
// t_end; stage 1 (prim, x/y/z faces, update, edge EMFs + CT in one pass): U^n -> S1;
// stage 2 (prim applies S1's deferred Joule sub-step in place): S1 -> S2;
// average: U^{n+1} = floors(0.5 (U^n + Joule(S2))) with the CFL partials of
// U^{n+1}; t += dt.  Three state buffers rotate; three steps are one CUDA graph.
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "checkpoint.h"
#include "handle.h"
#include "mhd3d_const.h"
#include "mhd3d_launch.h"

using namespace ccb;

namespace {

struct Mhd3dBase {
    virtual ~Mhd3dBase() {}
    virtual int init() = 0;
    virtual int upload(const double* const* f) = 0;
    virtual int download(double* const* f) = 0;
    virtual int compute_dt(double* dt) = 0;
    virtual int rk2_step(double dt) = 0;
    virtual int advance(int nsteps, double* t) = 0;
    virtual int diagnostics(cc_diag* d) = 0;
    virtual int derived(double* const* out) = 0;
    virtual int get_clock(double* t, long long* steps) = 0;
    virtual int set_clock(double t, long long steps) = 0;
    virtual const cc_mhd3d_params& params() const = 0;
};

template <class T> struct Mhd3d : Mhd3dBase {
    cc_handle* h;
    cc_mhd3d_params p;
    M3Const<T> c{};
    size_t vol = 0;          // elements of one pitched field
    void* block = nullptr;
    Fields3<T> buf[3];
    PrimData<T> prim{};
    Bcc3<T> bcc{};   // cell-centred B of the state a Joule pass reads
    FaceData<T> fX{}, fY{}, fZ{};
    double* staging = nullptr;
    double* spd_part = nullptr;
    double* rho_part = nullptr;
    double* diag_part = nullptr;
    double* scal = nullptr;   // dt, t
    long long* steps_dev = nullptr;
    int* iflags = nullptr;    // active
    double* derived_dev = nullptr;   // 11 planes of Nx*Ny*Nz, allocated at the first cc_mhd3d_derived
    int cur = 0;
    bool loaded = false;
    bool partials_valid = false;
    cudaGraphExec_t graph3 = nullptr;
    int graph_cur = -1;
    cudaStream_t graph_stream = nullptr;
    cc_perf graph_delta{};

    Mhd3d(cc_handle* hh, const cc_mhd3d_params& pp) : h(hh), p(pp) {}
    cc_handle* this_handle() { return h; }
    cudaStream_t st() const { return h->stream; }
    double* dt_dev() { return scal; }
    double* t_dev() { return scal + 1; }
    int* active() { return iflags; }
    void count(int n) { h->perf.kernel_launches += n; }

    ~Mhd3d() override {
        if (graph3) cudaGraphExecDestroy(graph3);
        void* ptrs[] = {block, staging, spd_part, rho_part, diag_part, scal, steps_dev, iflags, derived_dev};
        for (void* q : ptrs)
            if (q) cudaFree(q);
    }

    int init() override {
        const int nx = p.Nx, ny = p.Ny, nz = p.Nz;
        if ((long long)(nx + 1) * (ny + 1) * (nz + 1) >= (1ll << 31))
            return fail(h, CC_ERR_UNSUPPORTED, "3D grids need (Nx+1)(Ny+1)(Nz+1) < 2^31 (32-bit kernel indices)");
        c = m3_make_const<T>(p);
        vol = (size_t)c.PS * (nz + 1);

        // 3 states x 8 + primitives 8 + 3 x 7 face data + 3 cell-centred B = 56 fields
        const size_t nfield = 56;
        CC_CUDA(cudaMalloc(&block, sizeof(T) * vol * nfield));
        CC_CUDA(cudaMemsetAsync(block, 0, sizeof(T) * vol * nfield, st()));
        T* base = reinterpret_cast<T*>(block);
        auto take = [&]() { T* q = base; base += vol; return q; };
        for (int b = 0; b < 3; b++) {
            buf[b].rho = take(); buf[b].mx = take(); buf[b].my = take(); buf[b].mz = take(); buf[b].E = take();
            buf[b].bx = take(); buf[b].by = take(); buf[b].bz = take();
        }
        for (int m = 0; m < 8; m++) prim.w[m] = take();
        for (int m = 0; m < 7; m++) fX.f[m] = take();
        for (int m = 0; m < 7; m++) fY.f[m] = take();
        for (int m = 0; m < 7; m++) fZ.f[m] = take();
        bcc.x = take(); bcc.y = take(); bcc.z = take();
        CC_CUDA(cudaMalloc(&staging, sizeof(double) * (size_t)(nx + 1) * (ny + 1) * (nz + 1)));
        CC_CUDA(cudaMalloc(&spd_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&rho_part, sizeof(double) * RED_BLOCKS));
        CC_CUDA(cudaMalloc(&diag_part, sizeof(double) * RED_BLOCKS * 7));
        CC_CUDA(cudaMalloc(&scal, sizeof(double) * 4));
        CC_CUDA(cudaMemsetAsync(scal, 0, sizeof(double) * 4, st()));
        CC_CUDA(cudaMalloc(&steps_dev, sizeof(long long)));
        CC_CUDA(cudaMemsetAsync(steps_dev, 0, sizeof(long long), st()));
        CC_CUDA(cudaMalloc(&iflags, sizeof(int) * 4));
        int init_flags[4] = {1, 0, 0, 0};
        CC_CUDA(cudaMemcpyAsync(iflags, init_flags, sizeof(init_flags), cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    void dims(int k, int& w, int& hh, int& d) const {
        w = p.Nx + (k == 5); hh = p.Ny + (k == 6); d = p.Nz + (k == 7);
    }
    T* field(const Fields3<T>& f, int k) const {
        T* a[8] = {f.rho, f.mx, f.my, f.mz, f.E, f.bx, f.by, f.bz};
        return a[k];
    }

    int upload(const double* const* f) override {
        for (int k = 0; k < 8; k++) {
            if (!f[k]) return fail(h, CC_ERR_ARG, "null state array");
            int w, hh, d;
            dims(k, w, hh, d);
            CC_CUDA(cudaMemcpyAsync(staging, f[k], sizeof(double) * (size_t)w * hh * d, cudaMemcpyHostToDevice, st()));
            CC_CUDA(M3Launch<T>::pack_in(staging, field(buf[cur], k), w, hh, d, c.P, c.PS, st()));
            count(1);
        }
        loaded = true;
        partials_valid = false;
        return CC_OK;
    }

    int download(double* const* f) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        for (int k = 0; k < 8; k++) {
            if (!f[k]) continue;
            int w, hh, d;
            dims(k, w, hh, d);
            CC_CUDA(M3Launch<T>::pack_out(field(buf[cur], k), staging, w, hh, d, c.P, c.PS, st()));
            count(1);
            CC_CUDA(cudaMemcpyAsync(f[k], staging, sizeof(double) * (size_t)w * hh * d, cudaMemcpyDeviceToHost, st()));
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int ensure_partials() {
        if (partials_valid) return CC_OK;
        CC_CUDA(M3Launch<T>::speeds(c, buf[cur], spd_part, st()));
        count(1);
        partials_valid = true;
        return CC_OK;
    }

    DtSpec dtspec(bool clamp) const {
        const double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny, dz = (p.z1 - p.z0) / p.Nz;
        DtSpec d;
        d.cfl = p.cfl;
        d.hmin = vmin(vmin(dx, dy), dz);   // std::min({dx,dy,dz}) (M3:640)
        d.eta = p.eta;
        d.t_end = p.t_end;
        d.clamp_to_end = clamp ? 1 : 0;
        d.seed = 1e-14; d.end_eps = 0.0; d.check = 0; d.cap = 1;
        return d;
    }

    int compute_dt(double* dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        if (int r = ensure_partials()) return r;
        CC_CUDA(launch_dt_finalize(spd_part, dtspec(false), dt_dev(), t_dev(), active(), st()));
        count(1);
        CC_CUDA(cudaMemcpyAsync(dt, dt_dev(), sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    // one RK stage in -> out (M3:694-1030 without the Joule sub-step)
    int stage(const Fields3<T>& in, const Fields3<T>& out, bool defer) {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (h->profiling) {
            CC_CUDA(cudaEventCreate(&e0));
            CC_CUDA(cudaEventCreate(&e1));
            CC_CUDA(cudaEventRecord(e0, st()));
        }
        CC_CUDA(M3Launch<T>::prim(c, in, prim, defer, bcc, dt_dev(), active(), st()));
        CC_CUDA(M3Launch<T>::faces(c, in, prim, fX, fY, fZ, active(), st()));
        CC_CUDA(M3Launch<T>::update(c, in, out, fX, fY, fZ, dt_dev(), active(), st()));
        CC_CUDA(M3Launch<T>::emf_ct(c, in, out, fX, fY, fZ, dt_dev(), active(), st()));
        count(defer && c.resistive ? 7 : 6);
        if (h->profiling) {
            CC_CUDA(cudaEventRecord(e1, st()));
            h->timed.emplace_back(e0, e1);
        }
        return CC_OK;
    }

    int step_body() {
        const int a = cur, b = (cur + 1) % 3, d = (cur + 2) % 3;
        if (int r = stage(buf[a], buf[b], false)) return r;
        if (int r = stage(buf[b], buf[d], true)) return r;
        CC_CUDA(M3Launch<T>::average(c, buf[a], buf[d], buf[b], bcc, dt_dev(), active(), spd_part, rho_part, st()));
        count(c.resistive ? 2 : 1);
        h->perf.steps += 1;
        cur = b;
        partials_valid = true;
        return CC_OK;
    }

    int rk2_step(double dt) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        int one = 1;
        CC_CUDA(cudaMemcpyAsync(iflags, &one, sizeof(int), cudaMemcpyHostToDevice, st()));
        CC_CUDA(launch_set_scalar(dt_dev(), dt, st()));
        count(1);
        if (graph3) { cudaGraphExecDestroy(graph3); graph3 = nullptr; }
        if (int r = step_body()) return r;
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int device_step() {
        if (int r = ensure_partials()) return r;
        CC_CUDA(launch_dt_finalize(spd_part, dtspec(true), dt_dev(), t_dev(), active(), st()));
        count(1);
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
        if (int r = ensure_partials()) return r;
        int done = 0;
        if (!h->profiling && nsteps >= 3) {
            if (!graph3 || graph_cur != cur || graph_stream != st()) {
                if (graph3) { cudaGraphExecDestroy(graph3); graph3 = nullptr; }
                const int start = cur;
                const cc_perf before = h->perf;
                cudaGraph_t g = nullptr;
                CC_CUDA(cudaStreamBeginCapture(st(), cudaStreamCaptureModeThreadLocal));
                int rr = CC_OK;
                for (int k = 0; k < 3 && rr == CC_OK; k++) rr = device_step();
                cudaError_t e = cudaStreamEndCapture(st(), &g);
                cur = start;
                graph_delta.kernel_launches = h->perf.kernel_launches - before.kernel_launches;
                graph_delta.steps = h->perf.steps - before.steps;
                h->perf = before;
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
                h->perf.steps += graph_delta.steps;
                done += 3;
            }
            partials_valid = true;
        }
        for (; done < nsteps; ++done)
            if (int r = device_step()) return r;
        if (t) CC_CUDA(cudaMemcpyAsync(t, t_dev(), sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int derived(double* const* out) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        const size_t n = (size_t)p.Nx * p.Ny * p.Nz;
        if (!derived_dev) CC_CUDA(cudaMalloc(&derived_dev, sizeof(double) * n * 11));
        CC_CUDA(M3Launch<T>::derived(c, buf[cur], derived_dev, st()));
        for (int k = 0; k < 11; k++)
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

    const cc_mhd3d_params& params() const override { return p; }

    int diagnostics(cc_diag* d) override {
        if (!loaded) return fail(h, CC_ERR_STATE, "no state uploaded");
        CC_CUDA(M3Launch<T>::diag(c, buf[cur], diag_part, st()));
        count(1);
        std::vector<double> part(RED_BLOCKS * 7);
        CC_CUDA(cudaMemcpyAsync(part.data(), diag_part, sizeof(double) * part.size(), cudaMemcpyDeviceToHost, st()));
        double sc[4];
        CC_CUDA(cudaMemcpyAsync(sc, scal, sizeof(sc), cudaMemcpyDeviceToHost, st()));
        long long steps = 0;
        CC_CUDA(cudaMemcpyAsync(&steps, steps_dev, sizeof(steps), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        double s[5] = {0, 0, 0, 0, 0}, dmax = 0.0, nonf = 0.0;
        for (int m = 0; m < 5; m++)
            for (int b = 0; b < RED_BLOCKS; b++) s[m] += part[m * RED_BLOCKS + b];
        for (int b = 0; b < RED_BLOCKS; b++) {
            dmax = std::fmax(dmax, part[5 * RED_BLOCKS + b]);
            nonf = std::fmax(nonf, part[6 * RED_BLOCKS + b]);
        }
        const double dV = ((p.x1 - p.x0) / p.Nx) * ((p.y1 - p.y0) / p.Ny) * ((p.z1 - p.z0) / p.Nz);
        std::memset(d, 0, sizeof(*d));
        d->mass = s[0] * dV; d->mom_x = s[1] * dV; d->mom_y = s[2] * dV; d->mom_z = s[3] * dV; d->energy = s[4] * dV;
        d->max_divB = dmax;
        d->t = sc[1];
        d->dt_last = sc[0];
        d->steps = steps;
        d->nonfinite = nonf > 0.0 ? 1 : 0;
        return CC_OK;
    }
};

struct Mhd3dHandle : cc_handle {
    std::unique_ptr<Mhd3dBase> impl;
};

Mhd3dBase* m3(cc_handle* h) {
    if (!h || h->kind != KIND_MHD3D) return nullptr;
    return static_cast<Mhd3dHandle*>(h)->impl.get();
}

}  // namespace

extern "C" {

void cc_mhd3d_params_default(cc_mhd3d_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma1 = 1.30; p->gamma2 = 2.50; p->K1 = 0.05; p->rho_nuc = 80.0; p->gamma_th = 1.50;
    p->rho_bounce = 120.0; p->gamma_bounce = 3.00; p->Kbounce = 0.02; p->gamma_init = 5.0 / 3.0;
    p->cfl = 0.4;
    p->x0 = 0.0; p->x1 = 1.0; p->y0 = 0.0; p->y1 = 1.0; p->z0 = 0.0; p->z1 = 1.0;
    p->Nx = 48; p->Ny = 48; p->Nz = 48;
    p->precision = CC_FP64;
    p->t_end = 0.15; p->dt_store = 1e-3;
    p->floor_rho = 1e-10; p->floor_P = 1e-10;
    p->periodic_x = 1; p->periodic_y = 1; p->periodic_z = 1;
    p->eta = 5e-4;
}

int cc_mhd3d_create(const cc_mhd3d_params* p, cc_handle** out) {
    if (!p || !out) return CC_ERR_ARG;
    *out = nullptr;
    if (p->Nx < 2 || p->Ny < 2 || p->Nz < 2) return CC_ERR_ARG;
    if (!(p->x1 > p->x0) || !(p->y1 > p->y0) || !(p->z1 > p->z0)) return CC_ERR_ARG;
    if (p->precision != CC_FP64 && p->precision != CC_FP32) return CC_ERR_ARG;
    auto h = std::make_unique<Mhd3dHandle>();
    h->kind = KIND_MHD3D;
    if (cudaGetDevice(&h->device) != cudaSuccess) return CC_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return CC_ERR_CUDA;
    h->stream = h->own;
    if (p->precision == CC_FP64) h->impl = std::make_unique<Mhd3d<double>>(h.get(), *p);
    else h->impl = std::make_unique<Mhd3d<float>>(h.get(), *p);
    int r = h->impl->init();
    *out = h.release();
    return r;
}

int cc_mhd3d_upload(cc_handle* h, const double* rho, const double* mx, const double* my, const double* mz,
                    const double* E, const double* Bx_f, const double* By_f, const double* Bz_f) {
    Mhd3dBase* m = m3(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const double* f[8] = {rho, mx, my, mz, E, Bx_f, By_f, Bz_f};
    return m->upload(f);
}

int cc_mhd3d_download(cc_handle* h, double* rho, double* mx, double* my, double* mz, double* E, double* Bx_f,
                      double* By_f, double* Bz_f) {
    Mhd3dBase* m = m3(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    double* f[8] = {rho, mx, my, mz, E, Bx_f, By_f, Bz_f};
    return m->download(f);
}

int cc_mhd3d_compute_dt(cc_handle* h, double* dt) {
    Mhd3dBase* m = m3(h);
    if (!m || !dt) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->compute_dt(dt);
}

int cc_mhd3d_rk2_step(cc_handle* h, double dt) {
    Mhd3dBase* m = m3(h);
    if (!m) return CC_ERR_ARG;
    if (!std::isfinite(dt) || dt < 0.0) return fail(h, CC_ERR_NONFINITE, "dt not finite or negative");
    if (int r = set_dev(h)) return r;
    return m->rk2_step(dt);
}

int cc_mhd3d_advance(cc_handle* h, int nsteps, double* t) {
    Mhd3dBase* m = m3(h);
    if (!m) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->advance(nsteps, t);
}

int cc_mhd3d_diagnostics(cc_handle* h, cc_diag* d) {
    Mhd3dBase* m = m3(h);
    if (!m || !d) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->diagnostics(d);
}

int cc_mhd3d_derived(cc_handle* h, double* const* out) {
    Mhd3dBase* m = m3(h);
    if (!m || !out) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return m->derived(out);
}

// restart files (checkpoint.h): state {rho, mx, my, mz, E, Bx_f, By_f, Bz_f} and the clock
static std::vector<size_t> ck3_sizes_m3(const int32_t* n) {
    const size_t nx = (size_t)n[0], ny = (size_t)n[1], nz = (size_t)n[2], c = nx * ny * nz;
    return {c, c, c, c, c, (nx + 1) * ny * nz, nx * (ny + 1) * nz, nx * ny * (nz + 1)};
}

int cc_mhd3d_checkpoint_save(cc_handle* h, const char* path) {
    Mhd3dBase* m = m3(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_mhd3d_params& p = m->params();
    CkMeta meta;
    meta.precision = (uint32_t)p.precision;
    meta.n[0] = p.Nx; meta.n[1] = p.Ny; meta.n[2] = p.Nz;
    std::vector<std::vector<double>> f;
    for (size_t k : ck3_sizes_m3(meta.n)) f.emplace_back(k);
    double* fp[8];
    for (int k = 0; k < 8; k++) fp[k] = f[k].data();
    if (int r = m->download(fp)) return r;
    if (int r = m->get_clock(&meta.t, &meta.steps)) return r;
    std::string err;
    if (int r = ck3_save(path, "CCM3DCK1", meta, &p, sizeof(p), f, err)) return fail(h, r, err);
    return CC_OK;
}

int cc_mhd3d_checkpoint_load(cc_handle* h, const char* path) {
    Mhd3dBase* m = m3(h);
    if (!m || !path) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    const cc_mhd3d_params& p = m->params();
    CkMeta meta;
    cc_mhd3d_params q;
    std::vector<std::vector<double>> f;
    std::string err;
    if (int r = ck3_load(path, "CCM3DCK1", meta, &q, sizeof(q), ck3_sizes_m3, f, err)) return fail(h, r, err);
    if (meta.n[0] != p.Nx || meta.n[1] != p.Ny || meta.n[2] != p.Nz || (int)meta.precision != p.precision ||
        q.x0 != p.x0 || q.x1 != p.x1 || q.y0 != p.y0 || q.y1 != p.y1 || q.z0 != p.z0 || q.z1 != p.z1 ||
        q.periodic_x != p.periodic_x || q.periodic_y != p.periodic_y || q.periodic_z != p.periodic_z)
        return fail(h, CC_ERR_ARG, "checkpoint grid, domain, boundaries or precision differ from the handle's");
    const double* fp[8];
    for (int k = 0; k < 8; k++) fp[k] = f[k].data();
    if (int r = m->upload(fp)) return r;
    return m->set_clock(meta.t, meta.steps);
}

}  // extern "C"
