// Column-march form of the 2D MHD stage kernel (one RK stage of the reference,
// advance_stage M2:690-834, with the deferred Joule sub-step as in
// m2_stage_tile), used by the FP32 bulk path.
//
// A CTA owns a strip of W columns and a segment of rows, and marches up the
// segment R rows per step.  What the tile kernel recomputes in the y halo of
// every tile is carried from one step to the next in shared-memory rings
// indexed by the global row: the primitives (and the cells' own conserved
// state) of the two rows above the last update, the y slopes of one row, the
// x and y face fluxes of one row and the edge EMFs of one row.  So every x
// face, y face and edge of the strip is computed once (2.06 faces per cell
// instead of 2.32 for the 32 x 14 tile), and the primitives of 1.125 cells per
// cell (W + 4 columns) instead of 1.45.  Per step the threads take one round
// per phase: R x (W + 4) = NT primitives, then the x and y slopes (two
// rounds), the x and y faces (two rounds), the edges, the updates.
//
// A segment starts with a half step that builds the carried rows below its
// first row.  Every expression is the tile kernel's (same functions, same
// operands), so the FP32 result equals the tile kernel's up to the compiler's
// FMA contraction choices.
//
// KAHAN: compensated state as in m2_stage_tile (the cells' own residuals ride
// in a ring beside their conserved state).
#pragma once
#include "mhd2d_kernels.cuh"

namespace ccb {

template <class T, int W_, int R_> struct MarchGeom {
    static constexpr int W = W_, R = R_;
    static constexpr int PW = W + 4;    // primitive columns -2 .. W+1
    static constexpr int SW = W + 2;    // slope / y-face columns -1 .. W
    static constexpr int FW = W + 1;    // x faces / edges 0 .. W
    static constexpr int NPR = R + 2;   // primitive and own-state ring rows
    static constexpr int NFR = R + 1;   // y-slope, x-face, y-face and edge ring rows
    static constexpr int NT = (R * PW + 31) / 32 * 32;
    static_assert(NT >= R * SW && NT >= R * FW && NT >= R * W, "one round per phase");
    static constexpr size_t words(bool kahan) {
        return (size_t)8 * NPR * PW + (size_t)6 * NPR * W * (kahan ? 2 : 1) + (size_t)7 * R * SW +
               (size_t)7 * NFR * SW + (size_t)7 * NFR * FW + (size_t)7 * NFR * SW + (size_t)NFR * FW;
    }
    static constexpr size_t smem(bool kahan) { return sizeof(T) * words(kahan); }
};

// FP32 march shape: 32 columns, 8 rows a step, 288 threads, four CTAs per SM
constexpr int MARCH_W = 32, MARCH_R = 8, MARCH_MINB = 4;
using MarchG32 = MarchGeom<float, MARCH_W, MARCH_R>;

template <class T, int W, int R, bool DEFER, int GMODE, bool KAHAN>
__global__ void __launch_bounds__(MarchGeom<T, W, R>::NT, MARCH_MINB)
m2_march_kernel(const M2Const<T> c, const Fields<T> in, const Fields<T> out, const Fields<T> lin,
                const Fields<T> lout, const T* __restrict__ ga, const T* __restrict__ gb,
                const double* __restrict__ dtp, const int* __restrict__ active, const int seg_rows) {
    using G = MarchGeom<T, W, R>;
    constexpr int PW = G::PW, SW = G::SW, FW = G::FW, NPR = G::NPR, NFR = G::NFR, NT = G::NT;
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* const sm = reinterpret_cast<T*>(smem_raw);
    constexpr int PPL = NPR * PW;        // one primitive plane
    T* const s_r = sm;
    T* const s_u = s_r + PPL; T* const s_v = s_u + PPL; T* const s_w = s_v + PPL; T* const s_P = s_w + PPL;
    T* const s_bx = s_P + PPL; T* const s_by = s_bx + PPL; T* const s_bz = s_by + PPL;
    constexpr int OPL = NPR * W;         // one own-state plane
    T* const own = s_bz + PPL;           // 6 planes
    T* const own_lo = own + 6 * OPL;     // KAHAN: 6 planes
    constexpr int XPL = R * SW;          // one x-slope plane (rows of the current step)
    T* const xsl = own + 6 * OPL * (KAHAN ? 2 : 1);
    constexpr int YPL = NFR * SW;        // one y-slope / y-face plane
    T* const ysl = xsl + 7 * XPL;
    constexpr int FPL = NFR * FW;        // one x-face plane
    T* const fx = ysl + 7 * YPL;
    T* const gy = fx + 7 * FPL;
    T* const ez = gy + 7 * YPL;

    const int tid = threadIdx.x;
    const int P = c.pitch;
    const int i0 = blockIdx.x * W;
    const int jbeg = blockIdx.y * seg_rows;
    const int jend = min(jbeg + seg_rows, c.ny);
    const T dt = (T)(*dtp);
    // ring slots of a global row (rows >= -R - 2 here)
    auto ps = [](int g) { return (g + 8 * NPR) % NPR; };
    auto fs = [](int g) { return (g + 8 * NFR) % NFR; };
    auto pidx = [&](int g, int col) { return ps(g) * PW + col + 2; };   // col in -2 .. W+1

    // ---- primitives of rows [r0, r1) (get_prim_cc, M2:278-286), deferred Joule first ----
    auto prims = [&](int r0, int r1) {
        const int n = (r1 - r0) * PW;
        for (int k = tid; k < n; k += NT) {
            const int lr = k / PW, col = k - lr * PW - 2;
            const int g = r0 + lr;
            const int ci = c.ax.cell(i0 + col), cj = c.ay.cell(g);
            const size_t q = (size_t)cj * P + ci;
            T rho = in.rho[q], mx = in.mx[q], my = in.my[q], mz = in.mz[q], E = in.E[q], Bz = in.Bz[q];
            const T Bx = T(0.5) * (in.bx[q] + in.bx[q + 1]);
            const T By = T(0.5) * (in.by[q] + in.by[q + P]);
            const bool mine = col >= 0 && col < W;
            const int o = ps(g) * W + col;
            if constexpr (KAHAN) {
                if (mine) {
                    T h0 = rho, h4 = E, h5 = Bz;
                    T l0 = lin.rho[q], l4 = lin.E[q], l5 = lin.Bz[q];
                    if (DEFER) joule_cell_comp(c, in, ci, cj, dt, h0, l0, mx, my, mz, h4, l4, h5, l5, Bx, By);
                    own[o] = h0; own[OPL + o] = mx; own[2 * OPL + o] = my;
                    own[3 * OPL + o] = mz; own[4 * OPL + o] = h4; own[5 * OPL + o] = h5;
                    own_lo[o] = l0; own_lo[OPL + o] = lin.mx[q]; own_lo[2 * OPL + o] = lin.my[q];
                    own_lo[3 * OPL + o] = lin.mz[q]; own_lo[4 * OPL + o] = l4; own_lo[5 * OPL + o] = l5;
                }
            }
            if (DEFER) joule_cell(c, in, ci, cj, dt, rho, mx, my, mz, E, Bz, Bx, By);
            const Prim<T> Wp = to_prim(c, rho, mx, my, mz, E, Bx, By, Bz);
            const int kk = ps(g) * PW + col + 2;
            s_r[kk] = Wp.r; s_u[kk] = Wp.u; s_v[kk] = Wp.v; s_w[kk] = Wp.w;
            s_P[kk] = Wp.P; s_bx[kk] = Wp.bx; s_by[kk] = Wp.by; s_bz[kk] = Wp.bz;
            if (!KAHAN && mine) {
                own[o] = rho; own[OPL + o] = mx; own[2 * OPL + o] = my;
                own[3 * OPL + o] = mz; own[4 * OPL + o] = E; own[5 * OPL + o] = Bz;
            }
        }
    };

    // MC slopes of the seven reconstructed components of one cell along x
    // (M2:295-303): prims at ka - 1, ka, ka + 1; written at xsl[m * XPL + o]
    auto xslopes = [&](int ka, int o) {
        xsl[o] = mc_slope(s_r[ka - 1], s_r[ka], s_r[ka + 1]);
        xsl[XPL + o] = mc_slope(s_u[ka - 1], s_u[ka], s_u[ka + 1]);
        xsl[2 * XPL + o] = mc_slope(s_v[ka - 1], s_v[ka], s_v[ka + 1]);
        xsl[3 * XPL + o] = mc_slope(s_w[ka - 1], s_w[ka], s_w[ka + 1]);
        xsl[4 * XPL + o] = mc_slope(s_P[ka - 1], s_P[ka], s_P[ka + 1]);
        xsl[5 * XPL + o] = mc_slope(s_by[ka - 1], s_by[ka], s_by[ka + 1]);
        xsl[6 * XPL + o] = mc_slope(s_bz[ka - 1], s_bz[ka], s_bz[ka + 1]);
    };
    // face state of a cell: centre + side * 0.5 * slope, floored (M2:305-311)
    auto face_state = [&](int ka, const T* sl, int pl, int o, bool ydir, T side) {
        Prim<T> Wf;
        const T h = T(0.5) * side;
        Wf.r = s_r[ka] + h * sl[o];
        Wf.u = s_u[ka] + h * sl[pl + o];
        Wf.v = s_v[ka] + h * sl[2 * pl + o];
        Wf.w = s_w[ka] + h * sl[3 * pl + o];
        Wf.P = s_P[ka] + h * sl[4 * pl + o];
        if (ydir) { Wf.bx = s_bx[ka] + h * sl[5 * pl + o]; Wf.by = s_by[ka]; }
        else      { Wf.bx = s_bx[ka]; Wf.by = s_by[ka] + h * sl[5 * pl + o]; }
        Wf.bz = s_bz[ka] + h * sl[6 * pl + o];
        Wf.r = vmax(Wf.r, c.floor_rho);
        Wf.P = vmax(Wf.P, c.floor_P);
        return Wf;
    };

    // The first pass is a half step below the segment: primitives of rows
    // jbeg-2 .. jbeg+1, x and y slopes and x faces of rows jbeg-1, jbeg, the y
    // faces and edges of row jbeg.  Then each step from base row j computes
    // the primitives of rows [j+2, j+n+2), the x and y slopes and x faces of
    // rows [x0, x1) = [j+1, j+n+1), the y faces y and edges je in [y0, y1) =
    // [j+1, j+n+1), and updates rows [u0, u1) = [j, j+n).  (One loop, so
    // that the step body is inlined once.)
#pragma unroll 1
    for (int j = jbeg - R; j < jend; j += R) {
        const bool pre = j < jbeg;
        const int n = pre ? 0 : min(R, jend - j);
        const int p0 = pre ? jbeg - 2 : j + 2, p1 = pre ? jbeg + 2 : j + n + 2;
        const int x0 = pre ? jbeg - 1 : j + 1, x1 = pre ? jbeg + 1 : j + n + 1;
        const int y0 = pre ? jbeg : j + 1, y1 = pre ? jbeg + 1 : j + n + 1;
        const int u0 = j, u1 = j + n;
        prims(p0, p1);
        __syncthreads();
        {   // x and y slopes of rows [x0, x1) (ranges padded to whole warps)
            const int nx_ = (x1 - x0) * SW, nxp = (nx_ + 31) / 32 * 32, ny_ = (x1 - x0) * SW;
            for (int k = tid; k < nxp + ny_; k += NT) {
                if (k < nx_) {
                    const int lr = k / SW, col = k - lr * SW - 1;
                    xslopes(pidx(x0 + lr, col), lr * SW + col + 1);
                } else if (k >= nxp) {
                    const int kk = k - nxp;
                    const int lr = kk / SW, col = kk - lr * SW - 1;
                    const int g = x0 + lr;
                    const int ka = pidx(g, col);
                    // neighbours one row down / up in the ring (not a fixed stride; M2:319-327)
                    const int kd = pidx(g - 1, col), ku = pidx(g + 1, col);
                    const int o = fs(g) * SW + col + 1;
                    ysl[o] = mc_slope(s_r[kd], s_r[ka], s_r[ku]);
                    ysl[YPL + o] = mc_slope(s_u[kd], s_u[ka], s_u[ku]);
                    ysl[2 * YPL + o] = mc_slope(s_v[kd], s_v[ka], s_v[ku]);
                    ysl[3 * YPL + o] = mc_slope(s_w[kd], s_w[ka], s_w[ku]);
                    ysl[4 * YPL + o] = mc_slope(s_P[kd], s_P[ka], s_P[ku]);
                    ysl[5 * YPL + o] = mc_slope(s_bx[kd], s_bx[ka], s_bx[ku]);
                    ysl[6 * YPL + o] = mc_slope(s_bz[kd], s_bz[ka], s_bz[ku]);
                }
            }
        }
        __syncthreads();
        {   // x faces of rows [x0, x1) (M2:706-725), y faces y in [y0, y1) (M2:728-747)
            const int nx_ = (x1 - x0) * FW, nxp = (nx_ + 31) / 32 * 32, ny_ = (y1 - y0) * SW;
            for (int k = tid; k < nxp + ny_; k += NT) {
                if (k < nx_) {
                    const int lr = k / FW, f = k - lr * FW;
                    const int g = x0 + lr;
                    const int gi = i0 + f;
                    if (gi > c.nx) continue;
                    const int cj = c.ay.cell(g);
                    const Prim<T> WL = face_state(pidx(g, f - 1), xsl, XPL, lr * SW + f, false, T(1));
                    const Prim<T> WR = face_state(pidx(g, f), xsl, XPL, lr * SW + f + 1, false, T(-1));
                    const Flux<T> F = hlld_x(c, WL, WR, in.bx[(size_t)cj * P + gi]);
                    const int o = fs(g) * FW + f;
                    fx[o] = F.f0; fx[FPL + o] = F.f1; fx[2 * FPL + o] = F.f2; fx[3 * FPL + o] = F.f3;
                    fx[4 * FPL + o] = F.f4; fx[5 * FPL + o] = F.f5; fx[6 * FPL + o] = F.f6;
                } else if (k >= nxp) {
                    const int kk = k - nxp;
                    const int lr = kk / SW, col = kk - lr * SW - 1;
                    const int gj = y0 + lr;
                    if (gj > c.ny) continue;
                    const int ci = c.ax.cell(i0 + col);
                    const Prim<T> WL = face_state(pidx(gj - 1, col), ysl, YPL, fs(gj - 1) * SW + col + 1, true, T(1));
                    const Prim<T> WR = face_state(pidx(gj, col), ysl, YPL, fs(gj) * SW + col + 1, true, T(-1));
                    const Flux<T> Gf = hlld_y(c, WL, WR, in.by[(size_t)gj * P + ci]);
                    const int o = fs(gj) * SW + col + 1;
                    gy[o] = Gf.f0; gy[YPL + o] = Gf.f1; gy[2 * YPL + o] = Gf.f2; gy[3 * YPL + o] = Gf.f3;
                    gy[4 * YPL + o] = Gf.f4; gy[5 * YPL + o] = Gf.f5; gy[6 * YPL + o] = Gf.f6;
                }
            }
        }
        __syncthreads();
        // edge EMFs je in [y0, y1), ie = i0 .. i0 + W (M2:782-804, 565-575)
        for (int k = tid; k < (y1 - y0) * FW; k += NT) {
            const int lr = k / FW, e = k - lr * FW;
            const int ie = i0 + e, je = y0 + lr;
            if (ie > c.nx || je > c.ny) continue;
            const T exm = -fx[5 * FPL + fs(je - 1) * FW + e];   // x face ie, row je-1
            const T ex0 = -fx[5 * FPL + fs(je) * FW + e];       // x face ie, row je
            const T eym = gy[5 * YPL + fs(je) * SW + e];        // y face je, col ie-1
            const T ey0 = gy[5 * YPL + fs(je) * SW + e + 1];    // y face je, col ie
            const T ideal = T(0.25) * (exm + ex0 + eym + ey0);
            T res = T(0.0);
            if (c.resistive) {
                const int ci = c.ax.cell(ie), cim = c.ax.cell(ie - 1);
                const int cj = c.ay.cell(je), cjm = c.ay.cell(je - 1);
                const T dBydx = div_or_mul(in.by[(size_t)je * P + ci] - in.by[(size_t)je * P + cim], c.dx, c.inv_dx);
                const T dBxdy = div_or_mul(in.bx[(size_t)cj * P + ie] - in.bx[(size_t)cjm * P + ie], c.dy, c.inv_dy);
                res = c.eta * (dBydx - dBxdy);
            }
            ez[fs(je) * FW + e] = ideal + res;
        }
        __syncthreads();
        // FV update, floors, CT, gravity kick, store of rows [u0, u1) (M2:750-779, 807-832, 602-629)
        for (int k = tid; k < (u1 - u0) * W; k += NT) {
            const int lr = k / W, tx = k - lr * W;
            const int gi = i0 + tx, gj = u0 + lr;
            if (gi >= c.nx) continue;
            const size_t q = (size_t)gj * P + gi;
            const int o = ps(gj) * W + tx;
            T rho = own[o], mx = own[OPL + o], my = own[2 * OPL + o];
            T mz = own[3 * OPL + o], E = own[4 * OPL + o], Bz = own[5 * OPL + o];
            T lrho = T(0.0), lmx = T(0.0), lmy = T(0.0), lmz = T(0.0), lE = T(0.0), lBz = T(0.0);
            if constexpr (KAHAN) {
                lrho = own_lo[o]; lmx = own_lo[OPL + o]; lmy = own_lo[2 * OPL + o];
                lmz = own_lo[3 * OPL + o]; lE = own_lo[4 * OPL + o]; lBz = own_lo[5 * OPL + o];
            }
            const int fr = fs(gj) * FW + tx;                 // x faces tx, tx+1 of row gj
            const int gd = fs(gj) * SW + tx + 1, gu = fs(gj + 1) * SW + tx + 1;
            T d[7];
#pragma unroll
            for (int m = 0; m < 7; m++)
                d[m] = -(fx[m * FPL + fr + 1] - fx[m * FPL + fr]) * c.inv_dx -
                       (gy[m * YPL + gu] - gy[m * YPL + gd]) * c.inv_dy;
            const int kc = pidx(gj, tx);
            if constexpr (KAHAN) {
                comp_add(rho, lrho, dt * d[0]);
                comp_add(mx, lmx, dt * d[1]);
                comp_add(my, lmy, dt * d[2]);
                comp_add(mz, lmz, dt * d[3]);
                comp_add(E, lE, dt * d[4]);
                comp_add(Bz, lBz, dt * d[6]);
                floors_comp(c, rho, lrho, mx, my, mz, E, lE, s_bx[kc], s_by[kc], Bz);
            } else {
                rho += dt * d[0];
                mx += dt * d[1];
                my += dt * d[2];
                mz += dt * d[3];
                E += dt * d[4];
                Bz += dt * d[6];
                floors(c, rho, mx, my, mz, E, s_bx[kc], s_by[kc], Bz);
            }
            // CT (M2:807-830) for this cell's four faces
            const T dtdy = dt / c.dy, dtdx = dt / c.dx;
            const T e00 = ez[fs(gj) * FW + tx], e10 = ez[fs(gj) * FW + tx + 1];
            const T e01 = ez[fs(gj + 1) * FW + tx], e11 = ez[fs(gj + 1) * FW + tx + 1];
            T bxL, bxR, byD, byU;
            if constexpr (KAHAN) {
                T l0 = lin.bx[q], l1 = lin.bx[q + 1], l2 = lin.by[q], l3 = lin.by[q + P];
                bxL = in.bx[q]; bxR = in.bx[q + 1]; byD = in.by[q]; byU = in.by[q + P];
                comp_add(bxL, l0, -(dtdy) * (e01 - e00));
                comp_add(bxR, l1, -(dtdy) * (e11 - e10));
                comp_add(byD, l2, +(dtdx) * (e10 - e00));
                comp_add(byU, l3, +(dtdx) * (e11 - e01));
                lout.bx[q] = l0;
                if (gi == c.nx - 1) lout.bx[q + 1] = l1;
                lout.by[q] = l2;
                if (gj == c.ny - 1) lout.by[q + P] = l3;
            } else {
                bxL = in.bx[q] + -(dtdy) * (e01 - e00);
                bxR = in.bx[q + 1] + -(dtdy) * (e11 - e10);
                byD = in.by[q] + +(dtdx) * (e10 - e00);
                byU = in.by[q + P] + +(dtdx) * (e11 - e01);
            }
            out.bx[q] = bxL;
            if (gi == c.nx - 1) out.bx[q + 1] = bxR;
            out.by[q] = byD;
            if (gj == c.ny - 1) out.by[q + P] = byU;
            if (GMODE != GRAV_NONE && c.gravity_on) {
                T gxq, gyq;
                if (GMODE == GRAV_ARRAYS) {
                    gxq = ga[q]; gyq = gb[q];
                } else {
                    const T* phi = ga;
                    const int iE = c.ax.cell(gi + 1), iW = c.ax.cell(gi - 1);
                    const int jN = c.ay.cell(gj + 1), jS = c.ay.cell(gj - 1);
                    gxq = div_or_mul(-(phi[(size_t)gj * P + iE] - phi[(size_t)gj * P + iW]), c.two_dx,
                                     T(0.5) * c.inv_dx);
                    gyq = div_or_mul(-(phi[(size_t)jN * P + gi] - phi[(size_t)jS * P + gi]), c.two_dy,
                                     T(0.5) * c.inv_dy);
                }
                T u, v;
                if constexpr (fast_recip<T>()) {
                    const T ir = T(1.0) / vmax(rho, tiny_pos<T>());
                    u = mx * ir; v = my * ir;
                } else {
                    u = mx / vmax(rho, tiny_pos<T>());
                    v = my / vmax(rho, tiny_pos<T>());
                }
                if constexpr (KAHAN) {
                    comp_add(mx, lmx, dt * rho * gxq);
                    comp_add(my, lmy, dt * rho * gyq);
                    comp_add(E, lE, dt * rho * (u * gxq + v * gyq));
                    floors_comp(c, rho, lrho, mx, my, mz, E, lE, T(0.5) * (bxL + bxR), T(0.5) * (byD + byU), Bz);
                } else {
                    mx += dt * rho * gxq;
                    my += dt * rho * gyq;
                    E += dt * rho * (u * gxq + v * gyq);
                    floors(c, rho, mx, my, mz, E, T(0.5) * (bxL + bxR), T(0.5) * (byD + byU), Bz);
                }
            }
            out.rho[q] = rho; out.mx[q] = mx; out.my[q] = my; out.mz[q] = mz; out.E[q] = E; out.Bz[q] = Bz;
            if constexpr (KAHAN) {
                lout.rho[q] = lrho; lout.mx[q] = lmx; lout.my[q] = lmy; lout.mz[q] = lmz; lout.E[q] = lE;
                lout.Bz[q] = lBz;
            }
        }
        __syncthreads();
    }
}

}  // namespace ccb
