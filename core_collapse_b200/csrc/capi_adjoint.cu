// C ABI of the discrete adjoint of the 2D MHD step (include/cc_adjoint.h).
//
// A forward run of n steps (cc_adjoint_forward) keeps a checkpoint of the
// state every K steps and the dt of every step; cc_adjoint_vjp then walks the
// blocks of K steps backwards: each block is recomputed from its checkpoint
// with the recorded dt, storing what the reverse kernels need (stage inputs
// and outputs, potentials, stage records), and its steps are reversed one by
// one (adj2d_kernels.cuh).  dt is a recorded constant of the step (its
// dependence on the state through the CFL maximum is not differentiated), and
// gravity uses the direct Poisson solve, whose adjoint is the same solve
// (the discrete Laplacian is symmetric).
//
// Built with -fmad=false: the reverse kernels recompute forward intermediates
// (face states, floors, HLLD regions, limiter choices) and must round exactly
// like the FP64 forward kernels.
#include <memory>

#include "../../include/cc_adjoint.h"
#include "adj2d_kernels.cuh"
#include "batch_host.h"

using namespace ccb;

namespace {

constexpr int KIND_ADJOINT = 5;

int adj_grid(int n) {
    int g = (n + ADJ_NT - 1) / ADJ_NT;
    if (g > 148 * 8) g = 148 * 8;
    return g < 1 ? 1 : g;
}

struct Adjoint : Batch<double> {
    int K;
    int max_steps;
    int nrec = 0;                       // steps of the last recorded forward run
    std::vector<double> dts;            // host copy of the recorded dt
    double t0 = 0.0;
    double* dtrec = nullptr;
    double* lam_eta = nullptr;
    int P = 0;
    size_t plane = 0;
    bool grav = false;
    std::vector<Fields<double>> St, S1, S2, ckpt;
    std::vector<double*> Phi0, Phi1;
    std::vector<std::vector<double*>> Rec1, Rec2;
    Fields<double> fin{};
    Fields<double> LamA{}, LamB{}, LamS2{}, LamS1{}, LamIn{};
    double *LamB1x = nullptr, *LamB1y = nullptr, *LamBavx = nullptr, *LamBavy = nullptr;
    double *LamF5x = nullptr, *LamG5y = nullptr, *LamPhi = nullptr, *PoisOut = nullptr;
    double* LamD[6]{};
    double* LamW[8]{};
    double* Ut[6]{};
    double* Wp[8]{};
    double** dLamD = nullptr;
    double** dLamW = nullptr;
    double** dUt = nullptr;
    double** dWp = nullptr;
    std::vector<double**> dRec1, dRec2;
    BatchInst<double>* recA = nullptr;   // per local step: buf {St[l], S1[l], S2[l]}, phi Phi0[l], rec Rec1[l]
    BatchInst<double>* recB = nullptr;   // same buffers, phi Phi1[l], rec Rec2[l]
    BatchInst<double>* recC = nullptr;   // buf {St[l], St[l+1], S2[l]} for the average
    BatchInst<double>* recP = nullptr;   // Poisson adjoint: density <- LamPhi, phi -> PoisOut
    double** zAvg = nullptr;             // planes zeroed before the average reverse (LamS2, LamBav)
    double** zStage = nullptr;           // before a stage reverse (LamIn, LamW, LamF5x, LamG5y, LamPhi)
    double** zS1 = nullptr;              // LamS1
    bool loaded0 = false;

    Adjoint(cc_handle* hh, const cc_mhd2d_params& pp, int k, int mx)
        : Batch<double>(hh, &pp, 1), K(k), max_steps(mx) {}

    double* plane_alloc() {
        double* q = nullptr;
        if (dalloc(&q, plane) != CC_OK) return nullptr;
        if (cudaMemsetAsync(q, 0, sizeof(double) * plane, st()) != cudaSuccess) return nullptr;
        return q;
    }
    int state_alloc(Fields<double>& f) {
        double* q[8];
        for (int k = 0; k < 8; k++)
            if (!(q[k] = plane_alloc())) return fail(h, CC_ERR_CUDA, "device allocation failed");
        f = Fields<double>{q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7]};
        return CC_OK;
    }

    int init_adjoint() {
        if (int r = init()) return r;
        P = pitch[0];
        plane = (size_t)P * (p[0].Ny + 1);
        grav = p[0].gravity_on != 0;
        St.resize(K + 1); S1.resize(K); S2.resize(K);
        Phi0.resize(K); Phi1.resize(K);
        Rec1.assign(K, std::vector<double*>(6));
        Rec2.assign(K, std::vector<double*>(6));
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
        for (Fields<double>* f : {&LamA, &LamB, &LamS2, &LamS1, &LamIn})
            if (int r = state_alloc(*f)) return r;
        for (double** q : {&LamB1x, &LamB1y, &LamBavx, &LamBavy, &LamF5x, &LamG5y, &LamPhi, &PoisOut})
            if (!(*q = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
        for (int m = 0; m < 6; m++)
            if (!(LamD[m] = plane_alloc()) || !(Ut[m] = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
        for (int m = 0; m < 8; m++)
            if (!(LamW[m] = plane_alloc()) || !(Wp[m] = plane_alloc())) return fail(h, CC_ERR_CUDA, "alloc");
        std::vector<double*> v(LamD, LamD + 6);
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
            auto st8 = [](const Fields<double>& f, std::vector<double*>& v) {
                for (double* q : {f.rho, f.mx, f.my, f.mz, f.E, f.Bz, f.bx, f.by}) v.push_back(q);
            };
            std::vector<double*> za, zs, z1;
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
        std::vector<BatchInst<double>> A(K), B(K), C(K);
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
        std::vector<BatchInst<double>> Pv(1, hinst[0]);
        Pv[0].buf[0].rho = LamPhi;
        Pv[0].phi = PoisOut;
        if (int r = upload_vec(&recP, Pv)) return r;
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int copy_state(const Fields<double>& dst, const Fields<double>& src) {
        double* d[8] = {dst.rho, dst.mx, dst.my, dst.mz, dst.E, dst.Bz, dst.bx, dst.by};
        const double* s[8] = {src.rho, src.mx, src.my, src.mz, src.E, src.Bz, src.bx, src.by};
        for (int k = 0; k < 8; k++)
            CC_CUDA(cudaMemcpyAsync(d[k], s[k], sizeof(double) * plane, cudaMemcpyDeviceToDevice, st()));
        return CC_OK;
    }
    int zero_state(const Fields<double>& f) {
        double* d[8] = {f.rho, f.mx, f.my, f.mz, f.E, f.Bz, f.bx, f.by};
        for (int k = 0; k < 8; k++) CC_CUDA(cudaMemsetAsync(d[k], 0, sizeof(double) * plane, st()));
        return CC_OK;
    }
    int zero(double* q) {
        CC_CUDA(cudaMemsetAsync(q, 0, sizeof(double) * plane, st()));
        return CC_OK;
    }

    // host <-> device in the reference layouts (hin: upload; else download into hout)
    int xfer(const Fields<double>& f, const double* const* hin, double* const* hout) {
        const int nx = p[0].Nx, ny = p[0].Ny;
        const int w[8] = {nx, nx, nx, nx, nx, nx, nx + 1, nx};
        const int hh[8] = {ny, ny, ny, ny, ny, ny, ny, ny + 1};
        double* dev[8] = {f.rho, f.mx, f.my, f.mz, f.E, f.Bz, f.bx, f.by};
        for (int k = 0; k < 8; k++) {
            const size_t bytes = sizeof(double) * (size_t)w[k] * hh[k];
            if (hin) {
                if (!hin[k]) return fail(h, CC_ERR_ARG, "null array");
                CC_CUDA(cudaMemcpyAsync(staging, hin[k], bytes, cudaMemcpyHostToDevice, st()));
                CC_CUDA(M2Launch<double>::pack_in(staging, dev[k], w[k], hh[k], P, st()));
            } else {
                if (!hout[k]) continue;
                CC_CUDA(M2Launch<double>::pack_out(dev[k], staging, w[k], hh[k], P, st()));
                CC_CUDA(cudaMemcpyAsync(hout[k], staging, bytes, cudaMemcpyDeviceToHost, st()));
            }
        }
        CC_CUDA(cudaStreamSynchronize(st()));
        return CC_OK;
    }

    int upload0(const double* const* f) {
        if (int r = xfer(St[0], f, nullptr)) return r;
        loaded0 = true;   // the recorded dt sequence is kept: a replayed run may follow
        return CC_OK;
    }

    // mode 0: dt from the CFL condition (recorded); 1: recorded dt; 2: recorded dt + stage records
    int step(int l, int s, int mode) {
        const BatchInst<double>* A = recA + l;
        const BatchInst<double>* B = recB + l;
        const BatchInst<double>* Cc = recC + l;
        if (grav) {
            CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_MEAN, dt, tclk, active, rho_mean, st()));
            CC_CUDA(DPoissonLaunch<double>::solve(A, gwork, ngwork, gtile, nullptr, 0, ywork, nywork, 0, rho_mean,
                                                  active, tcerr, st()));
        }
        if (mode == 0) {
            CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_DT | BF_CLAMP, dt, tclk, active, rho_mean,
                                          st()));
            CC_CUDA(cudaMemcpyAsync(dtrec + s, dt, sizeof(double), cudaMemcpyDeviceToDevice, st()));
        } else {
            CC_CUDA(cudaMemcpyAsync(dt, dtrec + s, sizeof(double), cudaMemcpyDeviceToDevice, st()));
        }
        auto stage = [&](const BatchInst<double>* I, int src, int dst, bool defer) -> int {
            if (mode == 2)
                CC_CUDA(BatchLaunch<double>::stage_rec(I, swork[0], nswork[0], src, dst, defer, grav, dt, active, st()));
            else
                CC_CUDA(BatchLaunch<double>::stage(0, std::max(1, nswork[0]), I, swork[0], nswork[0], src, dst, defer,
                                                   grav, dt, active, st()));
            return CC_OK;
        };
        if (int r = stage(A, 0, 1, false)) return r;
        if (grav) {
            CC_CUDA(BatchLaunch<double>::rho_sum(B, rwork, nrwork, 1, active, rho_part, st()));
            CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_MEAN, dt, tclk, active, rho_mean, st()));
            CC_CUDA(DPoissonLaunch<double>::solve(B, gwork, ngwork, gtile, nullptr, 0, ywork, nywork, 1, rho_mean,
                                                  active, tcerr, st()));
        }
        if (int r = stage(B, 1, 2, true)) return r;
        CC_CUDA(BatchLaunch<double>::average(Cc, rwork, nrwork, 0, 2, 1, dt, active, spd_part, rho_part, st()));
        CC_CUDA(launch_batch_clock(1, tclk, dt, active, steps, st()));
        h->perf.kernel_launches += grav ? 13 : 5;
        h->perf.steps += 1;
        return CC_OK;
    }

    // steps [s0, s0 + L) from St[0]; mode as in step()
    int run_block(int s0, int L, int mode) {
        CC_CUDA(BatchLaunch<double>::speeds(recA, rwork, nrwork, 0, spd_part, rho_part, st()));
        for (int l = 0; l < L; l++)
            if (int r = step(l, s0 + l, mode)) return r;
        return CC_OK;
    }

    int forward(int nsteps, double tstart, int replay, double* tout) {
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

    int set_dts(const double* v, int n) {
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
    // LamPhi -> 4 pi G L^+ LamPhi (the same direct solve), added to ltarget.rho
    int poisson_adjoint(const Fields<double>& ltarget) {
        CC_CUDA(BatchLaunch<double>::rho_sum(recP, rwork, nrwork, 0, active, rho_part, st()));
        CC_CUDA(launch_batch_finalize(dred, 1, spd_part, rho_part, BF_MEAN, dt, tclk, active, rho_mean, st()));
        CC_CUDA(DPoissonLaunch<double>::solve(recP, gwork, ngwork, gtile, nullptr, 0, ywork, nywork, 0, rho_mean,
                                              active, tcerr, st()));
        adj_add_plane_kernel<<<adj_grid(p[0].Nx * p[0].Ny), ADJ_NT, 0, st()>>>(p[0].Nx, p[0].Ny, P, ltarget.rho,
                                                                                PoisOut);
        CC_CUDA(cudaGetLastError());
        h->perf.kernel_launches += 6;
        return CC_OK;
    }

    // one stage in reverse: lout (cells; its faces are lout.bx / lout.by) -> LamIn (zeroed here)
    int stage_reverse(const Fields<double>& sin, const Fields<double>& sout, const double* phi, double* const* drec,
                      bool defer, double dtv, const Fields<double>& lout) {
        const M2Const<double>& c = hinst[0].c;
        const int ncell = c.nx * c.ny;
        const int nedge = (c.nx + 1) * (c.ny + 1);
        adj_zero_kernel<<<adj_grid((int)(plane / 2)), ADJ_NT, 0, st()>>>(zStage, 19, plane);
        CC_CUDA(cudaGetLastError());
        CC_CUDA(cudaMemcpyAsync(LamB1x, lout.bx, sizeof(double) * plane, cudaMemcpyDeviceToDevice, st()));
        CC_CUDA(cudaMemcpyAsync(LamB1y, lout.by, sizeof(double) * plane, cudaMemcpyDeviceToDevice, st()));
        adj_prep_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, sin, defer, dtv, dUt, dWp);
        CC_CUDA(cudaGetLastError());
        adj_update_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, sin, sout, phi, drec, dtv, grav, lout, LamB1x,
                                                                LamB1y, LamIn, dLamD, LamPhi);
        CC_CUDA(cudaGetLastError());
        adj_edge_kernel<<<adj_grid(nedge), ADJ_NT, 0, st()>>>(c, sin, dtv, LamB1x, LamB1y, LamF5x, LamG5y, LamIn,
                                                              lam_eta);
        CC_CUDA(cudaGetLastError());
        adj_face_kernel<false><<<adj_grid((c.nx + 1) * c.ny), ADJ_NT, 0, st()>>>(c, sin, dWp, dLamD, LamF5x, dLamW,
                                                                                 LamIn);
        CC_CUDA(cudaGetLastError());
        adj_face_kernel<true><<<adj_grid(c.nx * (c.ny + 1)), ADJ_NT, 0, st()>>>(c, sin, dWp, dLamD, LamG5y, dLamW,
                                                                                LamIn);
        CC_CUDA(cudaGetLastError());
        adj_prim_kernel<<<adj_grid(ncell), ADJ_NT, 0, st()>>>(c, sin, dUt, dLamW, LamIn);
        CC_CUDA(cudaGetLastError());
        h->perf.kernel_launches += 6;
        return CC_OK;
    }

    // reverse of step s (local l): lnext (adjoint of St[l+1]) -> lun (adjoint of St[l])
    int step_reverse(int l, int s, const Fields<double>& lnext, const Fields<double>& lun) {
        const double dtv = dts[s];
        if (dtv == 0.0) return copy_state(lun, lnext);   // inactive step: identity
        const M2Const<double>& c = hinst[0].c;
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
            if (int r = poisson_adjoint(LamS1)) return r;
        // stage 1: U^n -> S1'
        if (int r = stage_reverse(St[l], S1[l], Phi0[l], dRec1[l], false, dtv, LamS1)) return r;
        adj_add_state_kernel<<<adj_grid(nedge), ADJ_NT, 0, st()>>>(c, lun, LamIn, true);
        CC_CUDA(cudaGetLastError());
        if (grav)
            if (int r = poisson_adjoint(lun)) return r;
        h->perf.kernel_launches += 5;
        return CC_OK;
    }

    int vjp(const double* const* lam_final, double* const* lam_init, double* eta_out) {
        if (nrec < 1) return fail(h, CC_ERR_STATE, "no recorded forward run");
        const int n = nrec;
        CC_CUDA(cudaMemsetAsync(lam_eta, 0, sizeof(double), st()));
        CC_CUDA(launch_batch_set_active(1, active, 1, st()));
        Fields<double> lnext = LamA, lun = LamB;
        if (int r = zero_state(lnext)) return r;
        if (int r = xfer(lnext, lam_final, nullptr)) return r;
        const int nb = (n + K - 1) / K;
        for (int b = nb - 1; b >= 0; b--) {
            const int s0 = b * K, L = std::min(K, n - s0);
            if (int r = copy_state(St[0], ckpt[b])) return r;
            if (int r = run_block(s0, L, 2)) return r;
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
};

struct AdjHandle : cc_handle {
    std::unique_ptr<Adjoint> impl;
};

Adjoint* aj(cc_handle* h) {
    if (!h || h->kind != KIND_ADJOINT) return nullptr;
    return static_cast<AdjHandle*>(h)->impl.get();
}

}  // namespace

extern "C" {

int cc_adjoint_create(const cc_mhd2d_params* p, int checkpoint_every, int max_steps, cc_handle** out) {
    if (!p || !out) return CC_ERR_ARG;
    *out = nullptr;
    auto h = std::make_unique<AdjHandle>();
    h->kind = KIND_ADJOINT;
    std::string why;
    int code = CC_OK;
    if (p->precision != CC_FP64) { code = CC_ERR_UNSUPPORTED; why = "the adjoint runs in FP64"; }
    else if (p->compensated) { code = CC_ERR_UNSUPPORTED; why = "the adjoint has no compensated update"; }
    else if (checkpoint_every < 1 || max_steps < 1) { code = CC_ERR_ARG; why = "checkpoint_every and max_steps must be >= 1"; }
    else if (p->Nx < 4 || p->Ny < 4 || !(p->x1 > p->x0) || !(p->y1 > p->y0)) { code = CC_ERR_ARG; why = "bad grid"; }
    else if (p->gravity_on && p->poisson_kind != CC_POISSON_DIRECT) {
        code = CC_ERR_UNSUPPORTED;
        why = "gravity needs poisson_kind == CC_POISSON_DIRECT (its adjoint is the same solve)";
    } else if (p->gravity_on && (p->Nx > CC_BATCH_MAX_DIRECT_SIDE || p->Ny > CC_BATCH_MAX_DIRECT_SIDE)) {
        code = CC_ERR_UNSUPPORTED;
        why = "direct Poisson side above CC_BATCH_MAX_DIRECT_SIDE";
    }
    if (code != CC_OK) {
        h->err = why;
        *out = h.release();
        return code;
    }
    if (cudaGetDevice(&h->device) != cudaSuccess) return CC_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return CC_ERR_CUDA;
    h->stream = h->own;
    cc_mhd2d_params q = *p;
    q.t_end = 1e300;   // the run length is the caller's step count
    h->impl = std::make_unique<Adjoint>(h.get(), q, checkpoint_every, max_steps);
    const int r = h->impl->init_adjoint();
    *out = h.release();
    return r;
}

int cc_adjoint_upload(cc_handle* h, const double* const* f) {
    Adjoint* a = aj(h);
    if (!a || !f) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->upload0(f);
}

int cc_adjoint_forward(cc_handle* h, int nsteps, double t0, int replay, double* t_out) {
    Adjoint* a = aj(h);
    if (!a) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->forward(nsteps, t0, replay, t_out);
}

int cc_adjoint_download(cc_handle* h, double* const* f) {
    Adjoint* a = aj(h);
    if (!a || !f) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->xfer(a->fin, nullptr, f);
}

int cc_adjoint_get_dts(cc_handle* h, double* dts, int n) {
    Adjoint* a = aj(h);
    if (!a || !dts || n < 0) return CC_ERR_ARG;
    if (n > a->nrec) return fail(h, CC_ERR_ARG, "fewer recorded steps than requested");
    for (int i = 0; i < n; i++) dts[i] = a->dts[i];
    return CC_OK;
}

int cc_adjoint_set_dts(cc_handle* h, const double* dts, int n) {
    Adjoint* a = aj(h);
    if (!a || !dts) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->set_dts(dts, n);
}

int cc_adjoint_vjp(cc_handle* h, const double* const* lam_final, double* const* lam_initial, double* lam_eta) {
    Adjoint* a = aj(h);
    if (!a || !lam_final) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->vjp(lam_final, lam_initial, lam_eta);
}

}  // extern "C"
