// The discrete adjoint of n steps of the 2D MHD solver, templated on the
// arithmetic type T of the forward run it reverses (include/cc_adjoint.h).
//
// A forward run of n steps (cc_adjoint_forward) keeps a checkpoint of the
// state every K steps and the dt of every step; cc_adjoint_vjp then walks the
// blocks of K steps backwards: each block is recomputed from its checkpoint
// with the recorded dt, storing what the reverse kernels need (stage inputs
// and outputs, potentials, stage records), and its steps are reversed one by
// one (adj2d_kernels.cuh).  dt is a recorded constant of the step (its
// dependence on the state through the CFL maximum is not differentiated), and
// gravity uses the direct Poisson solve, whose adjoint is the same solve
// (the discrete Laplacian is symmetric), or the red-black SOR of the single-
// grid solver with its recorded sweep count, reversed sweep by sweep
// (adj_sor_kernels.cuh).
//
// Instantiated for double in capi_adjoint.cu (-fmad=false: the reverse
// kernels recompute forward intermediates and must round like the FP64
// forward kernels) and for float in adjoint_f32.cu (the FP32 bulk-path flags
// of the FP32 forward kernels it recomputes).
#pragma once
#include <algorithm>
#include <initializer_list>
#include <vector>

#include "../../include/cc_adjoint.h"
#include "adj2d_kernels.cuh"
#include "adj_sor_kernels.cuh"
#include "mhd2d_launch.h"
#include "batch_host.h"

namespace ccb {

constexpr int KIND_ADJOINT = 5;

inline int adj_grid(int n) {
    int g = (n + ADJ_NT - 1) / ADJ_NT;
    if (g > 148 * 8) g = 148 * 8;
    return g < 1 ? 1 : g;
}

// what the C ABI calls, whatever the precision
struct AdjointBase {
    int nrec = 0;                       // steps of the last recorded forward run
    std::vector<double> dts;            // host copy of the recorded dt
    virtual ~AdjointBase() {}
    virtual int init_adjoint() = 0;
    virtual int upload0(const double* const* f) = 0;
    virtual int forward(int nsteps, double tstart, int replay, double* tout) = 0;
    virtual int download_final(double* const* f) = 0;
    virtual int set_dts(const double* v, int n) = 0;
    virtual int vjp(const double* const* lam_final, double* const* lam_init, double* eta_out) = 0;
};

template <class T> struct Adjoint : AdjointBase, Batch<T> {
    using B = Batch<T>;
    using B::h; using B::p; using B::pitch; using B::hinst; using B::dred; using B::rwork; using B::nrwork;
    using B::gwork; using B::ngwork; using B::gtile; using B::ywork; using B::nywork; using B::tcerr;
    using B::swork; using B::nswork; using B::spd_part; using B::rho_part; using B::dt; using B::tclk;
    using B::rho_mean; using B::active; using B::steps; using B::staging; using B::st; using B::dalloc;
    using B::upload_vec; using B::this_handle; using B::tcwork; using B::ntcwork;
    int K;
    int max_steps;
    double t0 = 0.0;
    double* dtrec = nullptr;
    double* lam_eta = nullptr;
    int P = 0;
    size_t plane = 0;
    bool grav = false;
    // red-black SOR gravity (poisson_kind CC_POISSON_SOR): forward solve
    // buffers, the sweep count of every solve (two per step), reverse buffers
    bool sor = false;
    double *srhs = nullptr, *sphi = nullptr, *spart = nullptr, *spart2 = nullptr, *sres = nullptr;
    double *smu0 = nullptr, *smu1 = nullptr, *srhat = nullptr, *sapart = nullptr;
    unsigned int* sbar = nullptr;
    int* sflags = nullptr;            // [barrier error, sweep count of the last solve]
    int* sor_iters_dev = nullptr;     // 2 per step
    std::vector<int> sor_iters_h;
    std::vector<Fields<T>> St, S1, S2, ckpt;
    std::vector<T*> Phi0, Phi1;
    std::vector<std::vector<T*>> Rec1, Rec2;
    Fields<T> fin{};
    Fields<T> LamA{}, LamB{}, LamS2{}, LamS1{}, LamIn{};
    T *LamB1x = nullptr, *LamB1y = nullptr, *LamBavx = nullptr, *LamBavy = nullptr;
    T *LamF5x = nullptr, *LamG5y = nullptr, *LamPhi = nullptr, *PoisOut = nullptr;
    T* LamD[6]{};
    T* LamW[8]{};
    T* Ut[6]{};
    T* Wp[8]{};
    T** dLamD = nullptr;
    T** dLamW = nullptr;
    T** dUt = nullptr;
    T** dWp = nullptr;
    std::vector<T**> dRec1, dRec2;
    BatchInst<T>* recA = nullptr;   // per local step: buf {St[l], S1[l], S2[l]}, phi Phi0[l], rec Rec1[l]
    BatchInst<T>* recB = nullptr;   // same buffers, phi Phi1[l], rec Rec2[l]
    BatchInst<T>* recC = nullptr;   // buf {St[l], St[l+1], S2[l]} for the average
    BatchInst<T>* recP = nullptr;   // Poisson adjoint: density <- LamPhi, phi -> PoisOut
    T** zAvg = nullptr;             // planes zeroed before the average reverse (LamS2, LamBav)
    T** zStage = nullptr;           // before a stage reverse (LamIn, LamW, LamF5x, LamG5y, LamPhi)
    T** zS1 = nullptr;              // LamS1
    bool loaded0 = false;

    Adjoint(cc_handle* hh, const cc_mhd2d_params& pp, int k, int mx)
        : Batch<T>(hh, &pp, 1), K(k), max_steps(mx) {}

    T* plane_alloc() {
        T* q = nullptr;
        if (dalloc(&q, plane) != CC_OK) return nullptr;
        if (cudaMemsetAsync(q, 0, sizeof(T) * plane, st()) != cudaSuccess) return nullptr;
        return q;
    }
    int state_alloc(Fields<T>& f) {
        T* q[8];
        for (int k = 0; k < 8; k++)
            if (!(q[k] = plane_alloc())) return fail(h, CC_ERR_CUDA, "device allocation failed");
        f = Fields<T>{q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]};
        return CC_OK;
    }

    int init_adjoint() override {
        if (int r = B::init()) return r;
        P = pitch[0];
        plane = (size_t)P * (p[0].Ny + 1);
        grav = p[0].gravity_on != 0;
        sor = grav && p[0].poisson_kind == CC_POISSON_SOR;
        if (sor) {
            const size_t N = (size_t)p[0].Nx * p[0].Ny;
            for (double** q : {&srhs, &sphi, &smu0, &smu1, &srhat})
                if (int r = dalloc(q, N)) return r;
            if (int r = dalloc(&spart, 4096)) return r;
            if (int r = dalloc(&spart2, 4096)) return r;
            if (int r = dalloc(&sapart, ASOR_BLOCKS)) return r;
            if (int r = dalloc(&sres, 1)) return r;
            if (int r = dalloc(&sbar, 2)) return r;
            if (int r = dalloc(&sflags, 2)) return r;
            if (int r = dalloc(&sor_iters_dev, 2 * (size_t)max_steps)) return r;
            CC_CUDA(cudaMemsetAsync(sbar, 0, sizeof(unsigned int) * 2, st()));
            CC_CUDA(cudaMemsetAsync(sflags, 0, sizeof(int) * 2, st()));
            sor_iters_h.assign(2 * (size_t)max_steps, 0);
        }
        St.resize(K + 1); S1.resize(K); S2.resize(K);
        Phi0.resize(K); Phi1.resize(K);
        Rec1.assign(K, std::vector<T*>(6));
        Rec2.assign(K, std::vector<T*>(6));
        for (int l = 0; l <= K; l++)
            if (int r = state_alloc(St[l])) return r;
        for (int l = 0; l < K; l++) {
            if (int r = state_alloc(S1[l])) return r;
            if (int r = state_alloc(S2[l])) return r;
            if (!(Phi0[l] = plane_alloc()) || !(Phi1[l] = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
            for (int m = 0; m < 6; m++)
                if (!(Rec1[l][m] = plane_alloc()) || !(Rec2[l][m] = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
        }
        const int nb = (max_steps + K - 1) / K + 1;
        ckpt.resize(nb);
        for (auto& f : ckpt)
            if (int r = state_alloc(f)) return r;
        if (int r = state_alloc(fin)) return r;
        {
            Fields<T>* const fs[5] = {&LamA, &LamB, &LamS2, &LamS1, &LamIn};
            for (int m = 0; m < 5; m++)
                if (int r = state_alloc(*fs[m])) return r;
        }
        {
            T** const qs[8] = {&LamB1x, &LamB1y, &LamBavx, &LamBavy, &LamF5x, &LamG5y, &LamPhi, &PoisOut};
            for (int m = 0; m < 8; m++)
                if (!(*qs[m] = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
        }
        for (int m = 0; m < 6; m++)
            if (!(LamD[m] = plane_alloc()) || !(Ut[m] = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
        for (int m = 0; m < 8; m++)
            if (!(LamW[m] = plane_alloc()) || !(Wp[m] = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
        std::vector<T*> v(LamD, LamD + 6);
        if (int r = upload_vec(&dLamD, v)) return r;
        v.assign(LamW, LamW + 8);
        if (int r = upload_vec(&dLamW, v)) return r;
        v.assign(Ut, Ut + 6);
        if (int r = upload_vec(&dUt, v)) return r;
        v.assign(Wp, Wp + 8);
        if (int r = upload_vec(&dWp, v)) return r;
        dRec1.resize(K); dRec2.resize(K);
        for (int l = 0; l < K; l++) {
            if (int r = upload_vec(&dRec1[l], Rec1[l])) return r;
            if (int r = upload_vec(&dRec2[l], Rec2[l])) return r;
        }
        {
            auto st8 = [](const Fields<T>& f, std::vector<T*>& v) {
                T* const a[8] = {f.rho, f.mx, f.my, f.mz, f.E, f.Bz, f.bx, f.by};
                for (int m = 0; m < 8; m++) v.push_back(a[m]);
            };
            std::vector<T*> za, zs, z1;
            st8(LamS2, za); za.push_back(LamBavx); za.push_back(LamBavy);
            st8(LamIn, zs); for (int m = 0; m < 8; m++) zs.push_back(LamW[m]);
            zs.push_back(LamF5x); zs.push_back(LamG5y); zs.push_back(LamPhi);
            st8(LamS1, z1);
            if (int r = upload_vec(&zAvg, za)) return r;
            if (int r = upload_vec(&zStage, zs)) return r;
            if (int r = upload_vec(&zS1, z1)) return r;
        }
        if (int r = dalloc(&dtrec, (size_t)max_steps)) return r;
        if (int r = dalloc(&lam_eta, 1)) return r;
        // record tables
        std::vector<BatchInst<T>> A(K), B(K), C(K);
        for (int l = 0; l < K; l++) {
            A[l] = hinst[0];
            A[l].buf[0] = St[l]; A[l].buf[1] = S1[l]; A[l].buf[2] = S2[l];
            A[l].phi = Phi0[l];
            for (int m = 0; m < 6; m++) A[l].rec[m] = Rec1[l][m];
            B[l] = A[l];
            B[l].phi = Phi1[l];
            for (int m = 0; m < 6; m++) B[l].rec[m] = Rec2[l][m];
            C[l] = A[l];
            C[l].buf[1] = St[l + 1];
        }
        if (int r = upload_vec(&recA, A)) return r;
        if (int r = upload_vec(&recB, B)) return r;
        if (int r = upload_vec(&recC, C)) return r;
        std::vector<BatchInst<T>> Pv(1, hinst[0]);
        Pv[0].buf[0].rho = LamPhi;
        Pv[0].phi = PoisOut;
        if (int r = upload_vec(&recP, Pv)) return r;
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int copy_state(const Fields<T>& dst, const Fields<T>& src) {
        T* d[8] = {dst.rho, dst.mx, dst.my, dst.mz, dst.E, dst.Bz, dst.bx, dst.by};
        const T* s[8] = {src.rho, src.mx, src.my, src.mz, src.E, src.Bz, src.bx, src.by};
        for (int k = 0; k < 8; k++)
            CC_CUDA(cudaMemcpyAsync(d[k], s[k], sizeof(T) * plane, cudaMemcpyDeviceToDevice, st()));
        return CC_OK;
    }
    int zero_state(const Fields<T>& f) {
        T* d[8] = {f.rho, f.mx, f.my, f.mz, f.E, f.Bz, f.bx, f.by};
        for (int k = 0; k < 8; k++) CC_CUDA(cudaMemsetAsync(d[k], 0, sizeof(T) * plane, st()));
        return CC_OK;
    }
    int zero(T* q) {
        CC_CUDA(cudaMemsetAsync(q, 0, sizeof(T) * plane, st()));
        return CC_OK;
    }

    // host <-> device in the reference layouts (hin: upload; else download into hout)
    int xfer(const Fields<T>& f, const double* const* hin, double* const* hout) {
        const int nx = p[0].Nx, ny = p[0].Ny;
        const int w[8] = {nx, nx, nx, nx, nx, nx, nx + 1, nx};
        const int hh[8] = {ny, ny, ny, ny, ny, ny, ny, ny + 1};
        T* dev[8] = {f.rho, f.mx, f.my, f.mz, f.E, f.Bz, f.bx, f.by};
        for (int k = 0; k < 8; k++) {
            const size_t bytes = sizeof(double) * (size_t)w[k] * hh[k];
            if (hin) {
                if (!hin[k]) return fail(h, CC_ERR_ARG, "null array");
                CC_CUDA(cudaMemcpyAsync(staging, hin[k], bytes, cudaMemcpyHostToDevice, st()));
                CC_CUDA(M2Launch<T>::pack_in(staging, dev[k], w[k], hh[k], P, st()));
            } else {
                if (!hout[k]) continue;
                CC_CUDA(M2Launch<T>::pack_out(dev[k], staging, w[k], hh[k], P, st()));
                CC_CUDA(cudaMemcpyAsync(hout[k], staging, bytes, cudaMemcpyDeviceToHost, st()));
            }
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int upload0(const double* const* f) override {
        if (int r = xfer(St[0], f, nullptr)) return r;
        loaded0 = true;   // the recorded dt sequence is kept: a replayed run may follow
        return CC_OK;
    }

    SorAdjArgs sor_adj_args() const {
        const double dx = (p[0].x1 - p[0].x0) / p[0].Nx, dy = (p[0].y1 - p[0].y0) / p[0].Ny;
        SorAdjArgs a;
        a.nx = p[0].Nx; a.ny = p[0].Ny;
        a.ax = AxisMap{p[0].Nx, p[0].periodic_x ? 1 : 0};
        a.ay = AxisMap{p[0].Ny, p[0].periodic_y ? 1 : 0};
        a.idx2 = 1.0 / (dx * dx); a.idy2 = 1.0 / (dy * dy);
        a.denom = 2.0 * (a.idx2 + a.idy2);
        a.omega = p[0].sor_omega;
        a.rhat = srhat; a.part = sapart;
        return a;
    }

    // forward red-black SOR of the density rho into the potential plane phi
    // (the single-grid solver's M2 solve: rhs from the density mean, phi = 0
    // start, sor_iters sweeps or the tolerance), its sweep count kept as
    // solve number `which`
    int sor_forward(const T* rho, T* phi, int which) {
        const int nx = p[0].Nx, ny = p[0].Ny;
        const int g = adj_grid(nx * ny);
        adj_sor_rhs_kernel<T><<<g, ADJ_NT, 0, st()>>>(rho, nx, ny, P, rho_mean, 4.0 * M_PI * p[0].G, srhs, active);
        CC_CUDA(cudaGetLastError());
        const SorAdjArgs b = sor_adj_args();
        SorArgs a;
        a.nx = nx; a.ny = ny; a.ax = b.ax; a.ay = b.ay;
        a.idx2 = b.idx2; a.idy2 = b.idy2; a.denom = b.denom;
        a.omega = p[0].sor_omega; a.tol = p[0].sor_tol; a.max_iter = p[0].sor_iters;
        a.rhs = srhs; a.phi = sphi; a.part = spart; a.part2 = spart2;
        a.bar = GridBarrier{sbar, sbar + 1, sflags};
        a.iters_out = sflags + 1; a.res_out = sres; a.active = active;
        int nb = 0;
        CC_CUDA(launch_sor(a, &nb, st()));
        phi_to_field_kernel<T><<<g, ADJ_NT, 0, st()>>>(sphi, nx, ny, phi, P, active);
        CC_CUDA(cudaGetLastError());
        CC_CUDA(cudaMemcpyAsync(sor_iters_dev + which, sflags + 1, sizeof(int), cudaMemcpyDeviceToDevice, st()));
        return CC_OK;
    }

    // host copy of the sweep counts of steps [s0, s0 + L); a timed-out grid barrier is an error
    int sor_counts(int s0, int L) {
        if (!sor) return CC_OK;
        int err = 0;
        CC_CUDA(cudaMemcpyAsync(&err, sflags, sizeof(int), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaMemcpyAsync(sor_iters_h.data() + 2 * s0, sor_iters_dev + 2 * s0, sizeof(int) * 2 * L,
                                cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        if (err) return fail(h, CC_ERR_CUDA, "SOR grid barrier timed out");
        return CC_OK;
    }

    // mode 0: dt from the CFL condition (recorded); 1: recorded dt; 2: recorded dt + stage records
    int step(int l, int s, int mode) {
        const BatchInst<T>* A = recA + l;
        const BatchInst<T>* B = recB + l;
        const BatchInst<T>* Cc = recC + l;
        if (grav) {
            CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_MEAN, dt, tclk, active, rho_mean, st()));
            if (sor) {
                if (int r = sor_forward(St[l].rho, Phi0[l], 2 * s)) return r;
            } else {
                CC_CUDA(DPoissonLaunch<T>::solve(A, gwork, ngwork, gtile, tcwork, ntcwork, ywork, nywork, 0, rho_mean,
                                                 active, tcerr, st()));
            }
        }
        if (mode == 0) {
            CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_DT | BF_CLAMP, dt, tclk, active, rho_mean,
                                          st()));
            CC_CUDA(cudaMemcpyAsync(dtrec + s, dt, sizeof(double), cudaMemcpyDeviceToDevice, st()));
        } else {
            CC_CUDA(cudaMemcpyAsync(dt, dtrec + s, sizeof(double), cudaMemcpyDeviceToDevice, st()));
        }
        auto stage = [&](const BatchInst<T>* I, int src, int dst, bool defer) -> int {
            if (mode == 2)
                CC_CUDA(BatchLaunch<T>::stage_rec(I, swork[0], nswork[0], src, dst, defer, grav, dt, active, st()));
            else
                CC_CUDA(BatchLaunch<T>::stage(0, std::max(1, nswork[0]), I, swork[0], nswork[0], src, dst, defer,
                                                   grav, dt, active, st()));
            return CC_OK;
        };
        if (int r = stage(A, 0, 1, false)) return r;
        if (grav) {
            CC_CUDA(BatchLaunch<T>::rho_sum(B, rwork, nrwork, 1, active, rho_part, st()));
            CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_MEAN, dt, tclk, active, rho_mean, st()));
            if (sor) {
                if (int r = sor_forward(S1[l].rho, Phi1[l], 2 * s + 1)) return r;
            } else {
                CC_CUDA(DPoissonLaunch<T>::solve(B, gwork, ngwork, gtile, tcwork, ntcwork, ywork, nywork, 1, rho_mean,
                                                 active, tcerr, st()));
            }
        }
        if (int r = stage(B, 1, 2, true)) return r;
        CC_CUDA(BatchLaunch<T>::average(Cc, rwork, nrwork, 0, 2, 1, dt, active, spd_part, rho_part, st()));
        CC_CUDA(launch_batch_clock(1, tclk, dt, active, steps, st()));
        h->perf.kernel_launches += grav ? 13 : 5;
        h->perf.steps += 1;
        return CC_OK;
    }

    // steps [s0, s0 + L) from St[0]; mode as in step()
    int run_block(int s0, int L, int mode) {
        CC_CUDA(BatchLaunch<T>::speeds(recA, rwork, nrwork, 0, spd_part, rho_part, st()));
        for (int l = 0; l < L; l++)
            if (int r = step(l, s0 + l, mode)) return r;
        return CC_OK;
    }

    int forward(int nsteps, double tstart, int replay, double* tout) override {
        if (!loaded0) return fail(h, CC_ERR_STATE, "no initial state uploaded");
        if (nsteps < 1 || nsteps > max_steps) return fail(h, CC_ERR_ARG, "nsteps outside [1, max_steps]");
        if (replay && nsteps > nrec) return fail(h, CC_ERR_STATE, "replay needs a recorded forward run of >= nsteps");
        t0 = tstart;
        CC_CUDA(cudaMemcpyAsync(tclk, &t0, sizeof(double), cudaMemcpyHostToDevice, st()));
        CC_CUDA(launch_batch_set_active(1, active, 1, st()));
        // St[0] holds the uploaded initial state; keep it in checkpoint 0
        if (int r = copy_state(ckpt[0], St[0])) return r;
        for (int s0 = 0, b = 0; s0 < nsteps; s0 += K, b++) {
            const int L = std::min(K, nsteps - s0);
            if (b > 0)
                if (int r = copy_state(St[0], ckpt[b])) return r;
            if (int r = run_block(s0, L, replay ? 1 : 0)) return r;
            if (int r = copy_state(ckpt[b + 1], St[L])) return r;
        }
        if (int r = copy_state(fin, ckpt[(nsteps + K - 1) / K])) return r;
        if (int r = copy_state(St[0], ckpt[0])) return r;   // initial state again, for the next run
        if (int r = sor_counts(0, nsteps)) return r;
        if (!replay) {
            nrec = nsteps;
            dts.assign(nsteps, 0.0);
            CC_CUDA(cudaMemcpyAsync(dts.data(), dtrec, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, st()));
        }
        double t = 0.0;
        CC_CUDA(cudaMemcpyAsync(&t, tclk, sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        if (tout) *tout = t;
        return CC_OK;
    }

    int set_dts(const double* v, int n) override {
        if (n < 1 || n > max_steps) return fail(h, CC_ERR_ARG, "n outside [1, max_steps]");
        for (int i = 0; i < n; i++)
            if (!(v[i] >= 0.0) || !std::isfinite(v[i])) return fail(h, CC_ERR_NONFINITE, "dt not finite or negative");
        dts.assign(v, v + n);
        CC_CUDA(cudaMemcpyAsync(dtrec, dts.data(), sizeof(double) * n, cudaMemcpyHostToDevice, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        nrec = n;
        return CC_OK;
    }

    // ---- reverse ----
    // SOR solve number `which` in reverse: LamPhi -> adjoint of its density, added to ltarget.rho
    int sor_adjoint(const Fields<T>& ltarget, int which) {
        const int K = sor_iters_h[which];
        const SorAdjArgs a = sor_adj_args();
        adj_sor_start_kernel<T><<<ASOR_BLOCKS, ASOR_NT, 0, st()>>>(a, LamPhi, P, smu0);
        CC_CUDA(cudaGetLastError());
        for (int k = 0; k < K; k++) {
            adj_sor_half_kernel<1, true, false><<<ASOR_BLOCKS, ASOR_NT, 0, st()>>>(a, smu0, smu1);
            adj_sor_half_kernel<0, false, true><<<ASOR_BLOCKS, ASOR_NT, 0, st()>>>(a, smu1, smu0);
        }
        CC_CUDA(cudaGetLastError());
        adj_sor_rhat_sum_kernel<ASOR_NT><<<ASOR_BLOCKS, ASOR_NT, 0, st()>>>(a);
        adj_sor_finish_kernel<T><<<ASOR_BLOCKS, ASOR_NT, 0, st()>>>(a, 4.0 * M_PI * p[0].G, ltarget.rho, P);
        CC_CUDA(cudaGetLastError());
        h->perf.kernel_launches += 3 + 2 * K;
        return CC_OK;
    }

    // LamPhi -> 4 pi G L^+ LamPhi (the same direct solve), added to ltarget.rho
    int poisson_adjoint(const Fields<T>& ltarget) {
        CC_CUDA(BatchLaunch<T>::rho_sum(recP, rwork, nrwork, 0, active, rho_part, st()));
        CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_MEAN, dt, tclk, active, rho_mean, st()));
        CC_CUDA(DPoissonLaunch<T>::solve(recP, gwork, ngwork, gtile, tcwork, ntcwork, ywork, nywork, 0, rho_mean,
                                              active, tcerr, st()));
        adj_add_plane_kernel<<<adj_grid(p[0].Nx * p[0].Ny), ADJ_NT, 0, st()>>>(p[0].Nx, p[0].Ny, P, ltarget.rho,
                                                                                PoisOut);
        CC_CUDA(cudaGetLastError());
        h->perf.kernel_launches += 6;
        return CC_OK;
    }

    // one stage in reverse: lout (cells; its faces are lout.bx / lout.by) -> LamIn (zeroed here)
    int stage_reverse(const Fields<T>& sin, const Fields<T>& sout, const T* phi, T* const* drec,
                      bool defer, T dtv, const Fields<T>& lout) {
        const M2Const<T>& c = hinst[0].c;
        const int ncell = c.nx * c.ny;
        const int nedge = (c.nx + 1) * (c.ny + 1);
        adj_zero_kernel<<<adj_grid((int)(plane / 2)), ADJ_NT, 0, st()>>>(zStage, 19, plane);
        CC_CUDA(cudaGetLastError());
        CC_CUDA(cudaMemcpyAsync(LamB1x, lout.bx, sizeof(T) * plane, cudaMemcpyDeviceToDevice, st()));
        CC_CUDA(cudaMemcpyAsync(LamB1y, lout.by, sizeof(T) * plane, cudaMemcpyDeviceToDevice, st()));
        adj_prep_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, sin, defer, dtv, dUt, dWp);
        CC_CUDA(cudaGetLastError());
        adj_update_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, sin, sout, phi, drec, dtv, grav, lout, LamB1x,
                                                                LamB1y, LamIn, dLamD, LamPhi);
        CC_CUDA(cudaGetLastError());
        adj_edge_kernel<<<adj_grid(nedge), ADJ_NT, 0, st()>>>(c, sin, dtv, LamB1x, LamB1y, LamF5x, LamG5y, LamIn,
                                                              lam_eta);
        CC_CUDA(cudaGetLastError());
        adj_face_kernel<T, false><<<adj_grid((c.nx + 1) * c.ny), ADJ_NT, 0, st()>>>(c, sin, dWp, dLamD, LamF5x, dLamW,
                                                                                 LamIn);
        CC_CUDA(cudaGetLastError());
        adj_face_kernel<T, true><<<adj_grid(c.nx * (c.ny + 1)), ADJ_NT, 0, st()>>>(c, sin, dWp, dLamD, LamG5y, dLamW,
                                                                                LamIn);
        CC_CUDA(cudaGetLastError());
        adj_prim_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, sin, dUt, dLamW, LamIn);
        CC_CUDA(cudaGetLastError());
        h->perf.kernel_launches += 6;
        return CC_OK;
    }

    // reverse of step s (local l): lnext (adjoint of St[l+1]) -> lun (adjoint of St[l])
    int step_reverse(int l, int s, const Fields<T>& lnext, const Fields<T>& lun) {
        const T dtv = (T)dts[s];
        if (dts[s] == 0.0) return copy_state(lun, lnext);   // inactive step: identity
        const M2Const<T>& c = hinst[0].c;
        const int ncell = c.nx * c.ny, nedge = (c.nx + 1) * (c.ny + 1);
        // RK average
        adj_zero_kernel<<<adj_grid((int)(plane / 2)), ADJ_NT, 0, st()>>>(zAvg, 10, plane);
        CC_CUDA(cudaGetLastError());
        adj_average_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, St[l], S2[l], dtv, lnext, lun, LamS2, LamBavx,
                                                                 LamBavy, lam_eta);
        CC_CUDA(cudaGetLastError());
        adj_average_face_kernel<<<adj_grid(nedge), ADJ_NT, 0, st()>>>(c, lnext, LamBavx, LamBavy, lun, LamS2);
        CC_CUDA(cudaGetLastError());
        // stage 2: Joule(S1') -> S2'
        if (int r = stage_reverse(S1[l], S2[l], Phi1[l], dRec2[l], true, dtv, LamS2)) return r;
        adj_zero_kernel<<<adj_grid((int)(plane / 2)), ADJ_NT, 0, st()>>>(zS1, 8, plane);
        CC_CUDA(cudaGetLastError());
        adj_joule_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, S1[l], dtv, LamIn, LamS1, lam_eta);
        CC_CUDA(cudaGetLastError());
        adj_add_state_kernel<<<adj_grid(nedge), ADJ_NT, 0, st()>>>(c, LamS1, LamIn, false);
        CC_CUDA(cudaGetLastError());
        if (grav)
            if (int r = sor ? sor_adjoint(LamS1, 2 * s + 1) : poisson_adjoint(LamS1)) return r;
        // stage 1: U^n -> S1'
        if (int r = stage_reverse(St[l], S1[l], Phi0[l], dRec1[l], false, dtv, LamS1)) return r;
        adj_add_state_kernel<<<adj_grid(nedge), ADJ_NT, 0, st()>>>(c, lun, LamIn, true);
        CC_CUDA(cudaGetLastError());
        if (grav)
            if (int r = sor ? sor_adjoint(lun, 2 * s) : poisson_adjoint(lun)) return r;
        h->perf.kernel_launches += 5;
        return CC_OK;
    }

    int vjp(const double* const* lam_final, double* const* lam_init, double* eta_out) override {
        if (nrec < 1) return fail(h, CC_ERR_STATE, "no recorded forward run");
        const int n = nrec;
        CC_CUDA(cudaMemsetAsync(lam_eta, 0, sizeof(double), st()));
        CC_CUDA(launch_batch_set_active(1, active, 1, st()));
        Fields<T> lnext = LamA, lun = LamB;
        if (int r = zero_state(lnext)) return r;
        if (int r = xfer(lnext, lam_final, nullptr)) return r;
        const int nb = (n + K - 1) / K;
        for (int b = nb - 1; b >= 0; b--) {
            const int s0 = b * K, L = std::min(K, n - s0);
            if (int r = copy_state(St[0], ckpt[b])) return r;
            if (int r = run_block(s0, L, 2)) return r;
            if (int r = sor_counts(s0, L)) return r;
            for (int l = L - 1; l >= 0; l--) {
                if (int r = step_reverse(l, s0 + l, lnext, lun)) return r;
                std::swap(lnext, lun);
            }
        }
        if (int r = copy_state(St[0], ckpt[0])) return r;
        if (lam_init)
            if (int r = xfer(lnext, nullptr, lam_init)) return r;
        if (eta_out) CC_CUDA(cudaMemcpyAsync(eta_out, lam_eta, sizeof(double), cudaMemcpyDeviceToHost, st()));
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int download_final(double* const* f) override { return xfer(fin, nullptr, f); }
};

}  // namespace ccb
