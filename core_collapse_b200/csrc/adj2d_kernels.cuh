// Discrete adjoint of one RK2 step of the 2D resistive-MHD solver, templated on
// the arithmetic type T of the forward it reverses (FP64, or FP32 with eta's
// adjoint accumulated in FP64).
//
// The forward step (mhd2d_kernels.cuh; M2:838-869) is
//   phi0 = P(U^n.rho)               S1' = Stage(U^n, phi0)        (pre-Joule)
//   phi1 = P(S1'.rho)               S2' = Stage(Joule(S1'), phi1)  (pre-Joule)
//   U^{n+1} = floors(0.5 (U^n + Joule(S2')))
// with Stage = halo prims -> MC slopes -> face states -> HLLD -> FV update +
// floors -> edge EMF -> CT -> gravity kick + floors, and dt a recorded
// constant.  Its adjoint is run backwards, one kernel per reverse sub-step,
// every forward intermediate needed being recomputed from the stored stage
// inputs / outputs and the stage record (the pre-floor update, REC variant of
// the stage tile), so every branch is the forward's.  Contributions that one
// thread scatters to cells or faces it does not own (slopes, face states,
// cell-centred B, the potential gradient, Joule neighbours, EMF averages) are
// atomic adds in T; eta's adjoint is block-reduced in FP64, then one atomic per block.
//
// Adjoint arrays share the pitched layout of the state (pitch P, ny+1 rows).
#pragma once
#include "mhd2d_adjoint.cuh"
#include "mhd2d_kernels.cuh"

namespace ccb {

constexpr int ADJ_NT = 256;

template <class T>
__device__ __forceinline__ void aadd(T* p, T v) {
    if (v != T(0)) atomicAdd(p, v);
}

__device__ __forceinline__ void eta_commit(double v, double* lam_eta) {
    __shared__ double sh[ADJ_NT / 32];
    const double b = block_sum<ADJ_NT>(v, sh);
    if (threadIdx.x == 0 && b != 0.0) atomicAdd(lam_eta, b);
}

// cell-centred B of a state at cell q (M2:278-286)
template <class T>
__device__ __forceinline__ T bxcc(const Fields<T>& s, size_t q) { return T(0.5) * (s.bx[q] + s.bx[q + 1]); }
template <class T>
__device__ __forceinline__ T bycc(const Fields<T>& s, size_t q, int P) {
    return T(0.5) * (s.by[q] + s.by[q + P]);
}

// Joule input of cell (i, j) of a stored stage output s (joule_cell's reads)
template <class T>
__device__ __forceinline__ JouleIn<T> joule_in(const M2Const<T>& c, const Fields<T>& s, int i, int j) {
    const int P = c.pitch;
    const size_t q = (size_t)j * P + i;
    const int iE = c.ax.cell(i + 1), iW = c.ax.cell(i - 1), jN = c.ay.cell(j + 1), jS = c.ay.cell(j - 1);
    JouleIn<T> J;
    J.rho = s.rho[q]; J.mx = s.mx[q]; J.my = s.my[q]; J.mz = s.mz[q]; J.E = s.E[q]; J.Bz = s.Bz[q];
    J.Bx = bxcc(s, q); J.By = bycc(s, q, P);
    J.bzE = s.Bz[(size_t)j * P + iE]; J.bzW = s.Bz[(size_t)j * P + iW];
    J.bzN = s.Bz[(size_t)jN * P + i]; J.bzS = s.Bz[(size_t)jS * P + i];
    J.byE = s.by[(size_t)j * P + iE]; J.byC = s.by[q];
    J.bxN = s.bx[(size_t)jN * P + i]; J.bxC = s.bx[q];
    return J;
}

// Scatter the adjoint of Joule's inputs at cell (i, j) into lam (a state-shaped adjoint).
template <class T>
__device__ __forceinline__ void joule_scatter(const M2Const<T>& c, const Fields<T>& lam, int i, int j,
                                              const JouleAdj<T>& a) {
    const int P = c.pitch;
    const size_t q = (size_t)j * P + i;
    const int iE = c.ax.cell(i + 1), iW = c.ax.cell(i - 1), jN = c.ay.cell(j + 1), jS = c.ay.cell(j - 1);
    aadd(lam.rho + q, a.l[0]); aadd(lam.mx + q, a.l[1]); aadd(lam.my + q, a.l[2]);
    aadd(lam.mz + q, a.l[3]); aadd(lam.E + q, a.l[4]); aadd(lam.Bz + q, a.l[5]);
    aadd(lam.Bz + (size_t)j * P + iE, a.bzE); aadd(lam.Bz + (size_t)j * P + iW, a.bzW);
    aadd(lam.Bz + (size_t)jN * P + i, a.bzN); aadd(lam.Bz + (size_t)jS * P + i, a.bzS);
    aadd(lam.by + (size_t)j * P + iE, a.byE); aadd(lam.by + q, a.byC + T(0.5) * a.By);
    aadd(lam.by + q + P, T(0.5) * a.By);
    aadd(lam.bx + (size_t)jN * P + i, a.bxN); aadd(lam.bx + q, a.bxC + T(0.5) * a.Bx);
    aadd(lam.bx + q + 1, T(0.5) * a.Bx);
}

// ---------------------------------------------------------------------------
// RK average (M2:848-868 with the deferred stage-2 Joule), reverse.
// lnext: adjoint of U^{n+1}; lun (cells, plain store), ls2 and lbavg (atomics).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(ADJ_NT)
adj_average_kernel(const M2Const<T> c, const Fields<T> un, const Fields<T> s2, T dt,
                   const Fields<T> lnext, const Fields<T> lun, const Fields<T> ls2,
                   T* __restrict__ lbavg_x, T* __restrict__ lbavg_y, double* __restrict__ lam_eta) {
    const int P = c.pitch;
    double leta = 0.0;
    for (int k = blockIdx.x * ADJ_NT + threadIdx.x; k < c.nx * c.ny; k += gridDim.x * ADJ_NT) {
        const int i = k % c.nx, j = k / c.nx;
        const size_t q = (size_t)j * P + i;
        // forward: Joule(S2') at this cell, then the average and floors
        const JouleIn<T> J = joule_in(c, s2, i, j);
        T rho = J.rho, mx = J.mx, my = J.my, mz = J.mz, E = J.E, Bz = J.Bz;
        joule_cell(c, s2, i, j, dt, rho, mx, my, mz, E, Bz, J.Bx, J.By);
        const T ar = T(0.5) * (un.rho[q] + rho), amx = T(0.5) * (un.mx[q] + mx), amy = T(0.5) * (un.my[q] + my);
        const T amz = T(0.5) * (un.mz[q] + mz), aE = T(0.5) * (un.E[q] + E), aBz = T(0.5) * (un.Bz[q] + Bz);
        const T bxl = T(0.5) * (un.bx[q] + s2.bx[q]), bxr = T(0.5) * (un.bx[q + 1] + s2.bx[q + 1]);
        const T byd = T(0.5) * (un.by[q] + s2.by[q]), byu = T(0.5) * (un.by[q + P] + s2.by[q + P]);
        const T Bx = T(0.5) * (bxl + bxr), By = T(0.5) * (byd + byu);
        T l0 = lnext.rho[q], l1 = lnext.mx[q], l2 = lnext.my[q], l3 = lnext.mz[q], l4 = lnext.E[q];
        T l5 = lnext.Bz[q], lBx = 0.0, lBy = 0.0;
        floors_vjp(c, ar, amx, amy, amz, aE, Bx, By, aBz, l0, l1, l2, l3, l4, lBx, lBy, l5);
        aadd(lbavg_x + q, T(0.5) * lBx); aadd(lbavg_x + q + 1, T(0.5) * lBx);
        aadd(lbavg_y + q, T(0.5) * lBy); aadd(lbavg_y + q + P, T(0.5) * lBy);
        lun.rho[q] = T(0.5) * l0; lun.mx[q] = T(0.5) * l1; lun.my[q] = T(0.5) * l2;
        lun.mz[q] = T(0.5) * l3; lun.E[q] = T(0.5) * l4; lun.Bz[q] = T(0.5) * l5;
        JouleAdj<T> a{};
        a.l[0] = T(0.5) * l0; a.l[1] = T(0.5) * l1; a.l[2] = T(0.5) * l2; a.l[3] = T(0.5) * l3; a.l[4] = T(0.5) * l4; a.l[5] = T(0.5) * l5;
        if (c.resistive) joule_vjp(c, dt, J, a);
        joule_scatter(c, ls2, i, j, a);
        leta += a.eta;
    }
    eta_commit(leta, lam_eta);
}

// faces of the average: B^{n+1} = 0.5 (B^n + B2'); lbavg holds the floors' share
template <class T>
__global__ void adj_average_face_kernel(const M2Const<T> c, const Fields<T> lnext,
                                        const T* __restrict__ lbavg_x, const T* __restrict__ lbavg_y,
                                        const Fields<T> lun, const Fields<T> ls2) {
    const int P = c.pitch;
    const int n = (c.nx + 1) * (c.ny + 1);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = k % (c.nx + 1), j = k / (c.nx + 1);
        const size_t q = (size_t)j * P + i;
        if (j < c.ny) {   // Bx face (i, j), i <= nx
            const T l = T(0.5) * (lnext.bx[q] + lbavg_x[q]);
            lun.bx[q] = l;
            ls2.bx[q] += l;
        }
        if (i < c.nx) {   // By face (i, j), j <= ny
            const T l = T(0.5) * (lnext.by[q] + lbavg_y[q]);
            lun.by[q] = l;
            ls2.by[q] += l;
        }
    }
}

// ---------------------------------------------------------------------------
// Stage reverse, step A: stage inputs after the deferred Joule (ut) and their
// primitives (wp), recomputed once per cell.
// ---------------------------------------------------------------------------
template <class T>
__global__ void adj_prep_kernel(const M2Const<T> c, const Fields<T> sin, bool defer, T dt,
                                T* const* ut, T* const* wp) {
    const int P = c.pitch;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < c.nx * c.ny; k += gridDim.x * blockDim.x) {
        const int i = k % c.nx, j = k / c.nx;
        const size_t q = (size_t)j * P + i;
        T rho = sin.rho[q], mx = sin.mx[q], my = sin.my[q], mz = sin.mz[q], E = sin.E[q], Bz = sin.Bz[q];
        const T Bx = bxcc(sin, q), By = bycc(sin, q, P);
        if (defer) joule_cell(c, sin, i, j, dt, rho, mx, my, mz, E, Bz, Bx, By);
        ut[0][q] = rho; ut[1][q] = mx; ut[2][q] = my; ut[3][q] = mz; ut[4][q] = E; ut[5][q] = Bz;
        const Prim<T> W = to_prim(c, rho, mx, my, mz, E, Bx, By, Bz);
        wp[0][q] = W.r; wp[1][q] = W.u; wp[2][q] = W.v; wp[3][q] = W.w;
        wp[4][q] = W.P; wp[5][q] = W.bx; wp[6][q] = W.by; wp[7][q] = W.bz;
    }
}

// ---------------------------------------------------------------------------
// Stage reverse, step B (cells): final floors + gravity kick (M2:602-629),
// then the update floors (M2:777) and the update itself.
// lout: adjoint of the stage output (cells; its faces are lb1 below).
// lb1: adjoint of the output faces, += the final floors' share (atomics).
// lin: adjoint of the stage input (after Joule): cells and faces (atomics).
// ld: dt * adjoint of the pre-floor update (plain store, 6 planes).
// lphi: adjoint of the potential (atomics).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(ADJ_NT)
adj_update_kernel(const M2Const<T> c, const Fields<T> sin, const Fields<T> sout,
                  const T* __restrict__ phi, const T* const* rec, T dt, bool grav,
                  const Fields<T> lout, T* __restrict__ lb1x, T* __restrict__ lb1y,
                  const Fields<T> lin, T* const* ld, T* __restrict__ lphi) {
    const int P = c.pitch;
    for (int k = blockIdx.x * ADJ_NT + threadIdx.x; k < c.nx * c.ny; k += gridDim.x * ADJ_NT) {
        const int i = k % c.nx, j = k / c.nx;
        const size_t q = (size_t)j * P + i;
        // forward: the pre-floor update, its floors with the stage-input B
        const T rr = rec[0][q], rmx = rec[1][q], rmy = rec[2][q], rmz = rec[3][q], rE = rec[4][q];
        const T rBz = rec[5][q];
        const T Bx0 = bxcc(sin, q), By0 = bycc(sin, q, P);
        T rho = rr, E = rE;
        floors(c, rho, rmx, rmy, rmz, E, Bx0, By0, rBz);
        T l0 = lout.rho[q], l1 = lout.mx[q], l2 = lout.my[q], l3 = lout.mz[q], l4 = lout.E[q], l5 = lout.Bz[q];
        if (grav && c.gravity_on) {
            const int iE = c.ax.cell(i + 1), iW = c.ax.cell(i - 1), jN = c.ay.cell(j + 1), jS = c.ay.cell(j - 1);
            const T gx = -(phi[(size_t)j * P + iE] - phi[(size_t)j * P + iW]) / c.two_dx;
            const T gy = -(phi[(size_t)jN * P + i] - phi[(size_t)jS * P + i]) / c.two_dy;
            const T rv = vmax(rho, tiny_pos<T>());
            const T u = rmx / rv, v = rmy / rv;
            const T kmx = rmx + dt * rho * gx, kmy = rmy + dt * rho * gy;
            const T kE = E + dt * rho * (u * gx + v * gy);
            const T B1x = bxcc(sout, q), B1y = bycc(sout, q, P);
            T lBx = 0.0, lBy = 0.0;
            floors_vjp(c, rho, kmx, kmy, rmz, kE, B1x, B1y, rBz, l0, l1, l2, l3, l4, lBx, lBy, l5);
            aadd(lb1x + q, T(0.5) * lBx); aadd(lb1x + q + 1, T(0.5) * lBx);
            aadd(lb1y + q, T(0.5) * lBy); aadd(lb1y + q + P, T(0.5) * lBy);
            // kick (rho, mz, Bz pass through)
            const T lkmx = l1, lkmy = l2, lkE = l4;
            l0 += dt * gx * lkmx + dt * gy * lkmy + dt * (u * gx + v * gy) * lkE;
            const T lu = dt * rho * gx * lkE, lv = dt * rho * gy * lkE;
            const T lgx = dt * rho * lkmx + dt * rho * u * lkE;
            const T lgy = dt * rho * lkmy + dt * rho * v * lkE;
            l1 = lkmx + lu / rv;
            l2 = lkmy + lv / rv;
            if (!(rho < tiny_pos<T>())) l0 -= (lu * u + lv * v) / rv;
            aadd(lphi + (size_t)j * P + iE, -lgx / c.two_dx);
            aadd(lphi + (size_t)j * P + iW, lgx / c.two_dx);
            aadd(lphi + (size_t)jN * P + i, -lgy / c.two_dy);
            aadd(lphi + (size_t)jS * P + i, lgy / c.two_dy);
        }
        // update floors with the stage-input B
        T lBx = 0.0, lBy = 0.0;
        floors_vjp(c, rr, rmx, rmy, rmz, rE, Bx0, By0, rBz, l0, l1, l2, l3, l4, lBx, lBy, l5);
        aadd(lin.bx + q, T(0.5) * lBx); aadd(lin.bx + q + 1, T(0.5) * lBx);
        aadd(lin.by + q, T(0.5) * lBy); aadd(lin.by + q + P, T(0.5) * lBy);
        // U1 = Ut + dt d
        aadd(lin.rho + q, l0); aadd(lin.mx + q, l1); aadd(lin.my + q, l2);
        aadd(lin.mz + q, l3); aadd(lin.E + q, l4); aadd(lin.Bz + q, l5);
        ld[0][q] = dt * l0; ld[1][q] = dt * l1; ld[2][q] = dt * l2;
        ld[3][q] = dt * l3; ld[4][q] = dt * l4; ld[5][q] = dt * l5;
    }
}

// ---------------------------------------------------------------------------
// Stage reverse, step C (edges (nx+1) x (ny+1)): CT (M2:807-830) and the edge
// EMF (M2:782-804, 565-575).  Each edge thread also passes the output-face
// adjoint through CT to the input face it owns (Bx face (ie, je), By face
// (ie, je)).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(ADJ_NT)
adj_edge_kernel(const M2Const<T> c, const Fields<T> sin, T dt, const T* __restrict__ lb1x,
                const T* __restrict__ lb1y, T* __restrict__ lf5x, T* __restrict__ lg5y,
                const Fields<T> lin, double* __restrict__ lam_eta) {
    const int P = c.pitch;
    const T dtdy = dt / c.dy, dtdx = dt / c.dx;
    double leta = 0.0;
    const int n = (c.nx + 1) * (c.ny + 1);
    for (int k = blockIdx.x * ADJ_NT + threadIdx.x; k < n; k += gridDim.x * ADJ_NT) {
        const int ie = k % (c.nx + 1), je = k / (c.nx + 1);
        T lez = 0.0;
        if (je < c.ny) lez += dtdy * lb1x[(size_t)je * P + ie];
        if (je >= 1) lez -= dtdy * lb1x[(size_t)(je - 1) * P + ie];
        if (ie < c.nx) lez -= dtdx * lb1y[(size_t)je * P + ie];
        if (ie >= 1) lez += dtdx * lb1y[(size_t)je * P + ie - 1];
        // pass-through B1 = Bin + ...
        if (je < c.ny) aadd(lin.bx + (size_t)je * P + ie, lb1x[(size_t)je * P + ie]);
        if (ie < c.nx) aadd(lin.by + (size_t)je * P + ie, lb1y[(size_t)je * P + ie]);
        if (lez == 0.0) continue;
        const int cj = c.ay.cell(je), cjm = c.ay.cell(je - 1), ci = c.ax.cell(ie), cim = c.ax.cell(ie - 1);
        aadd(lf5x + (size_t)cjm * P + ie, T(-0.25) * lez);
        aadd(lf5x + (size_t)cj * P + ie, T(-0.25) * lez);
        aadd(lg5y + (size_t)je * P + cim, T(0.25) * lez);
        aadd(lg5y + (size_t)je * P + ci, T(0.25) * lez);
        if (c.resistive) {
            const T dBydx = (sin.by[(size_t)je * P + ci] - sin.by[(size_t)je * P + cim]) / c.dx;
            const T dBxdy = (sin.bx[(size_t)cj * P + ie] - sin.bx[(size_t)cjm * P + ie]) / c.dy;
            leta += lez * (dBydx - dBxdy);
            const T e = c.eta * lez;
            aadd(lin.by + (size_t)je * P + ci, e / c.dx);
            aadd(lin.by + (size_t)je * P + cim, -e / c.dx);
            aadd(lin.bx + (size_t)cj * P + ie, -e / c.dy);
            aadd(lin.bx + (size_t)cjm * P + ie, e / c.dy);
        }
    }
    eta_commit(leta, lam_eta);
}

// face-state reconstruction (M2:295-311) of one side of a face, reverse:
// scatter the adjoint of the floored face state lf (7 reconstructed
// components, prim planes comp[k]) into lw at the mapped cells.
template <class T>
__device__ __forceinline__ void face_state_scatter(const M2Const<T>& c, T* const* wp, T* const* lw,
                                                   const int comp[7], size_t qm, size_t q0, size_t qp, T h,
                                                   const T lf[7]) {
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const int m = comp[k];
        const T wm = wp[m][qm], wc = wp[m][q0], wq = wp[m][qp];
        const T s = mc_slope(wm, wc, wq);
        T l = lf[k];
        if (k == 0 && (wc + h * s) < c.floor_rho) l = 0.0;   // r = vmax(r, floor_rho)
        if (k == 4 && (wc + h * s) < c.floor_P) l = 0.0;     // P = vmax(P, floor_P)
        if (l == 0.0) continue;
        T lm = 0.0, lc = l, lp = 0.0;
        mc_slope_vjp(wm, wc, wq, h * l, lm, lc, lp);
        aadd(lw[m] + qm, lm);
        aadd(lw[m] + q0, lc);
        aadd(lw[m] + qp, lp);
    }
}

template <class T>
__device__ __forceinline__ Prim<T> face_state_fwd(const M2Const<T>& c, T* const* wp, size_t qm,
                                                       size_t q0, size_t qp, T h, bool ydir) {
    Prim<T> W;
    T v[8];
#pragma unroll
    for (int m = 0; m < 8; m++) v[m] = wp[m][q0];
    const int rc[7] = {0, 1, 2, 3, 4, ydir ? 5 : 6, 7};
#pragma unroll
    for (int k = 0; k < 7; k++) {
        const int m = rc[k];
        v[m] = wp[m][q0] + h * mc_slope(wp[m][qm], wp[m][q0], wp[m][qp]);
    }
    W.r = vmax(v[0], c.floor_rho); W.u = v[1]; W.v = v[2]; W.w = v[3]; W.P = vmax(v[4], c.floor_P);
    W.bx = v[5]; W.by = v[6]; W.bz = v[7];
    return W;
}

// ---------------------------------------------------------------------------
// Stage reverse, step D: x faces (nx+1) x ny, or y faces nx x (ny+1).
// Face flux adjoint from the update (ld of the two cells) and the EMF (lf5),
// then HLLD, face states and MC slopes in reverse; lw (primitive adjoints)
// and the normal-B adjoint of the input face by atomics.
// ---------------------------------------------------------------------------
template <class T, bool YDIR>
__global__ void __launch_bounds__(ADJ_NT)
adj_face_kernel(const M2Const<T> c, const Fields<T> sin, T* const* wp, T* const* ld,
                const T* __restrict__ lf5, T* const* lw, const Fields<T> lin) {
    const int P = c.pitch;
    const int nf = YDIR ? c.nx * (c.ny + 1) : (c.nx + 1) * c.ny;
    const int rc[7] = {0, 1, 2, 3, 4, YDIR ? 5 : 6, 7};
    for (int k = blockIdx.x * ADJ_NT + threadIdx.x; k < nf; k += gridDim.x * ADJ_NT) {
        int f, r;   // face index along the normal, and the line (row for x, column for y)
        if (!YDIR) { f = k % (c.nx + 1); r = k / (c.nx + 1); }
        else { r = k % c.nx; f = k / c.nx; }
        const AxisMap& ax = YDIR ? c.ay : c.ax;
        const int nn = YDIR ? c.ny : c.nx;
        auto cq = [&](int pos) -> size_t {
            const int m = ax.cell(pos);
            return YDIR ? (size_t)m * P + r : (size_t)r * P + m;
        };
        const size_t qLm = cq(f - 2), qL = cq(f - 1), qR = cq(f), qRp = cq(f + 1);
        const size_t qface = YDIR ? (size_t)f * P + r : (size_t)r * P + f;
        // flux adjoint: d(cell) = -(F(face+1) - F(face)) / h; ld = dt * adj(U1raw)
        const T ih = YDIR ? c.inv_dy : c.inv_dx;
        T lF[7];
        const int dmap[7] = {0, 1, 2, 3, 4, -1, 5};
#pragma unroll
        for (int m = 0; m < 7; m++) {
            if (dmap[m] < 0) { lF[m] = lf5[qface]; continue; }
            T v = 0.0;
            if (f < nn) v += ld[dmap[m]][YDIR ? (size_t)f * P + r : (size_t)r * P + f];
            if (f >= 1) v -= ld[dmap[m]][YDIR ? (size_t)(f - 1) * P + r : (size_t)r * P + f - 1];
            lF[m] = ih * v;
        }
        bool any = false;
#pragma unroll
        for (int m = 0; m < 7; m++) any = any || (lF[m] != 0.0);
        if (!any) continue;
        Flux<T> g;
        g.f0 = lF[0]; g.f1 = lF[1]; g.f2 = lF[2]; g.f3 = lF[3]; g.f4 = lF[4]; g.f5 = lF[5]; g.f6 = lF[6];
        const Prim<T> WL = face_state_fwd(c, wp, qLm, qL, qR, T(0.5), YDIR);
        const Prim<T> WR = face_state_fwd(c, wp, qL, qR, qRp, T(-0.5), YDIR);
        const T Bn = YDIR ? sin.by[qface] : sin.bx[qface];
        Prim<T> lL = prim_zero<T>(), lR = prim_zero<T>();
        T lBn = 0.0;
        if (YDIR) hlld_y_vjp(c, WL, WR, Bn, g, lL, lR, lBn);
        else hlld_x_vjp(c, WL, WR, Bn, g, lL, lR, lBn);
        aadd((YDIR ? lin.by : lin.bx) + qface, lBn);
        const T aL[8] = {lL.r, lL.u, lL.v, lL.w, lL.P, lL.bx, lL.by, lL.bz};
        const T aR[8] = {lR.r, lR.u, lR.v, lR.w, lR.P, lR.bx, lR.by, lR.bz};
        T fl[7], fr[7];
#pragma unroll
        for (int m = 0; m < 7; m++) { fl[m] = aL[rc[m]]; fr[m] = aR[rc[m]]; }
        face_state_scatter(c, wp, lw, rc, qLm, qL, qR, T(0.5), fl);
        face_state_scatter(c, wp, lw, rc, qL, qR, qRp, T(-0.5), fr);
    }
}

// ---------------------------------------------------------------------------
// Stage reverse, step E (cells): primitives (M2:126-135) in reverse.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(ADJ_NT)
adj_prim_kernel(const M2Const<T> c, const Fields<T> sin, T* const* ut, T* const* lw,
                const Fields<T> lin) {
    const int P = c.pitch;
    for (int k = blockIdx.x * ADJ_NT + threadIdx.x; k < c.nx * c.ny; k += gridDim.x * ADJ_NT) {
        const int i = k % c.nx, j = k / c.nx;
        const size_t q = (size_t)j * P + i;
        Prim<T> l;
        l.r = lw[0][q]; l.u = lw[1][q]; l.v = lw[2][q]; l.w = lw[3][q];
        l.P = lw[4][q]; l.bx = lw[5][q]; l.by = lw[6][q]; l.bz = lw[7][q];
        T a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, aBx = 0, aBy = 0, aBz = 0;
        to_prim_vjp(c, ut[0][q], ut[1][q], ut[2][q], ut[3][q], ut[4][q], bxcc(sin, q), bycc(sin, q, P), ut[5][q], l,
                    a0, a1, a2, a3, a4, aBx, aBy, aBz);
        aadd(lin.rho + q, a0); aadd(lin.mx + q, a1); aadd(lin.my + q, a2);
        aadd(lin.mz + q, a3); aadd(lin.E + q, a4); aadd(lin.Bz + q, aBz);
        aadd(lin.bx + q, T(0.5) * aBx); aadd(lin.bx + q + 1, T(0.5) * aBx);
        aadd(lin.by + q, T(0.5) * aBy); aadd(lin.by + q + P, T(0.5) * aBy);
    }
}

// ---------------------------------------------------------------------------
// Stage-2 input: Ut = Joule(S1') (deferred Joule, M2:631-686), reverse.
// lin: adjoint of Ut (cells) and of the input faces; ls1 += adjoint of S1'.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(ADJ_NT)
adj_joule_kernel(const M2Const<T> c, const Fields<T> s1, T dt, const Fields<T> lin,
                 const Fields<T> ls1, double* __restrict__ lam_eta) {
    const int P = c.pitch;
    double leta = 0.0;
    for (int k = blockIdx.x * ADJ_NT + threadIdx.x; k < c.nx * c.ny; k += gridDim.x * ADJ_NT) {
        const int i = k % c.nx, j = k / c.nx;
        const size_t q = (size_t)j * P + i;
        JouleAdj<T> a{};
        a.l[0] = lin.rho[q]; a.l[1] = lin.mx[q]; a.l[2] = lin.my[q];
        a.l[3] = lin.mz[q]; a.l[4] = lin.E[q]; a.l[5] = lin.Bz[q];
        if (c.resistive) joule_vjp(c, dt, joule_in(c, s1, i, j), a);
        joule_scatter(c, ls1, i, j, a);
        leta += a.eta;
    }
    eta_commit(leta, lam_eta);
}

// dst += src over the cells (if `cells`) and faces of a state-shaped adjoint
template <class T>
__global__ void adj_add_state_kernel(const M2Const<T> c, const Fields<T> dst, const Fields<T> src,
                                     bool cells) {
    const int P = c.pitch;
    const int n = (c.nx + 1) * (c.ny + 1);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const int i = k % (c.nx + 1), j = k / (c.nx + 1);
        const size_t q = (size_t)j * P + i;
        if (cells && i < c.nx && j < c.ny) {
            dst.rho[q] += src.rho[q]; dst.mx[q] += src.mx[q]; dst.my[q] += src.my[q];
            dst.mz[q] += src.mz[q]; dst.E[q] += src.E[q]; dst.Bz[q] += src.Bz[q];
        }
        if (j < c.ny) dst.bx[q] += src.bx[q];
        if (i < c.nx) dst.by[q] += src.by[q];
    }
}

// zero nplanes planes of `plane` values each (one launch for a whole set)
template <class T>
__global__ void adj_zero_kernel(T* const* planes, int nplanes, size_t plane) {
    for (int k = 0; k < nplanes; k++) {
        T* q = planes[k];
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < plane; i += (size_t)gridDim.x * blockDim.x)
            q[i] = T(0);
    }
}

// dst[q] += src[q] over the cells of a pitched plane
template <class T>
__global__ void adj_add_plane_kernel(int nx, int ny, int P, T* __restrict__ dst, const T* __restrict__ src) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nx * ny; k += gridDim.x * blockDim.x) {
        const size_t q = (size_t)(k / nx) * P + (k % nx);
        dst[q] += src[q];
    }
}

}  // namespace ccb
