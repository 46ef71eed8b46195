// 2D resistive-MHD step kernels (templated on T; instantiated per precision in
// mhd2d_f64.cu / mhd2d_f32.cu).
//
// Device layout: every field is a pitched 2D array with the same pitch P
// (elements, multiple of 32) and ny+1 rows:
//   cells  c[j*P + i]          i < nx,  j < ny
//   Bx     bx[j*P + i_face]    i_face <= nx, j < ny
//   By     by[j_face*P + i]    i < nx, j_face <= ny
//
// One RK stage of the reference (advance_stage, M2:690-834) is ONE kernel here:
// a CTA owns a TX x TY tile of cells, builds primitives on a halo-2 region in
// shared memory, computes the x and y HLLD face fluxes it needs, the FV update,
// the edge EMFs, the CT face update and the gravity kick, and writes the stage
// output.  The reference's last sub-step, Joule heating + Bz diffusion + floors
// (M2:631-686), needs post-update Bz of neighbouring cells; instead of a second
// pass it is applied lazily by whichever kernel next reads the stage output
// (the stage-2 prologue, and the RK-average kernel), from the stored pre-Joule
// state.  Because that function depends only on global arrays addressed with
// the reference's own wrap rules, the value every reader computes for a cell is
// the reference's value, also across the periodic seam where the reference's
// face arrays wrap modulo N+1.
#pragma once
#include "mhd2d_physics.cuh"

namespace ccb {

template <class T> struct Fields {
    T* rho; T* mx; T* my; T* mz; T* E; T* Bz; T* bx; T* by;
};

enum GravMode { GRAV_NONE = 0, GRAV_ARRAYS = 1, GRAV_PHI = 2 };

// Stage tile per precision: TX x TY cells per CTA, NT threads, a halo-2
// region of primitives, one shared slope buffer reused for x then y.  Every
// phase is a loop of its items over the NT threads between two barriers, so
// a phase whose item count is just above NT costs a second, nearly empty
// round while the CTA's other warps wait at the barrier.  The FP32 tile is
// sized so that slopes, x faces, y faces, edges and cells each fit one round
// and each warp works one row of a phase (ROW32): 30 x 15 cells, 544 threads
// = 17 rows of 32 slope cells, 17 rows of 31 x faces, 16 rows of 32 y faces.
// FP64 the same way on 30 x 8 cells and 320 threads (10 rows of slopes).
// Measured against 32 x 14 / 32 x 8 tiles with warps across row ends: FP32
// stage 1.281 -> 1.196 ms, FP64 5.71 -> 4.55 ms at 4096^2.
// SPLIT: separate x and y slope buffers (7 NSL more shared memory), so that
// the x and y slopes form one phase and the x and y face fluxes another
// (4 barriers per tile instead of 6; each item range padded to whole warps so
// no warp mixes x and y work).
template <class T> struct StageTile;
template <> struct StageTile<double> {
    static constexpr int TX = 30, TY = 8, NT = 320, MINB = 2;
    static constexpr bool SPLIT = false;
};
template <> struct StageTile<float> {
    static constexpr int TX = 30, TY = 15, NT = 544, MINB = 2;
    static constexpr bool SPLIT = false;
};

template <class T, int TX_, int TY_, int NT_ = TX_ * TY_, bool SPLIT_ = false> struct StageGeomT {
    static constexpr int TX = TX_, TY = TY_, HALO = 2;
    static constexpr int RX = TX + 2 * HALO, RY = TY + 2 * HALO, RR = RX * RY;
    static constexpr int NT = NT_;        // threads
    static constexpr int NC = TX * TY;    // cells
    static constexpr bool SPLIT = SPLIT_;
    // ROW32: a tile TX = 30 wide, so that slope and y-face rows are 32 items
    // wide; x faces, edges and cells are then also mapped one row per warp
    // (a lane per column, the last lanes idle), so no warp straddles two rows
    // and the shared-memory reads of a phase hit 32 distinct banks
    static constexpr bool ROW32 = (TX + 2 == 32);
    // ROWSYNC: one warp per slope row (NT = 32 (TY + 2) threads).  A warp then
    // writes the x slopes of its row, reads them for the x faces of the same
    // row and writes the y slopes of that row into the same slots: no other
    // warp touches them, so these phases are separated by __syncwarp only;
    // likewise its y-face row and then its edge row
    static constexpr bool ROWSYNC = ROW32 && NT == 32 * (TY + 2);
    static_assert(NT >= NC && NT % 32 == 0, "one thread per cell in the update phase, whole warps");
    static_assert(!ROW32 || (32 * TY <= NT && !SPLIT), "ROW32: a row of threads per tile row of cells, no split");
    static constexpr int NFX = (TX + 1) * (TY + 2);  // x faces: TX+1 per row, rows -1..TY
    static constexpr int NGY = (TX + 2) * (TY + 1);  // y faces: cols -1..TX, TY+1 per col
    static constexpr int NE = (TX + 1) * (TY + 1);   // edges
    static constexpr int NSL = (TX + 2) * (TY + 2);  // cells whose slopes a face needs
    static constexpr int NSB = SPLIT ? 2 : 1;         // slope buffers
    // prims (8 RR) + slopes (7 NSL each) + x fluxes (7 NFX) + y fluxes (7 NGY) + Ez + own state (6 NC)
    static constexpr size_t smem = sizeof(T) * (size_t)(8 * RR + 7 * NSB * NSL + 7 * NFX + 7 * NGY + NE + 6 * NC);
};

template <class T>
using StageGeom = StageGeomT<T, StageTile<T>::TX, StageTile<T>::TY, StageTile<T>::NT, StageTile<T>::SPLIT>;
template <class T> constexpr size_t m2_stage_smem() { return StageGeom<T>::smem; }

// Joule heating, explicit Bz diffusion and floors of one cell
// (add_joule_heating_and_Bz_resistive, M2:631-686), applied to the stored
// pre-Joule state s at cell (i,j); the cell's own values are passed in and
// E, Bz, rho are updated.  Bx, By are the cell-centred stage-output B.
// |J|^2 and the 5-point Laplacian of Bz of cell (i,j) of the stored state s,
// whose own Bz is bzC (M2:640-668)
template <class T>
__device__ __forceinline__ void joule_terms(const M2Const<T>& c, const Fields<T>& s, int i, int j, T bzC, T& J2,
                                            T& lap) {
    const int P = c.pitch;
    const int iE = c.ax.cell(i + 1), iW = c.ax.cell(i - 1);
    const int jN = c.ay.cell(j + 1), jS = c.ay.cell(j - 1);
    const T bzE = s.Bz[(size_t)j * P + iE], bzW = s.Bz[(size_t)j * P + iW];
    const T bzN = s.Bz[(size_t)jN * P + i], bzS = s.Bz[(size_t)jS * P + i];
    const T dBzdy = div_or_mul(bzN - bzS, c.two_dy, T(0.5) * c.inv_dy);
    const T dBzdx = div_or_mul(bzE - bzW, c.two_dx, T(0.5) * c.inv_dx);
    const T dBydx = div_or_mul(s.by[(size_t)j * P + iE] - s.by[(size_t)j * P + i], c.dx, c.inv_dx);
    const T dBxdy = div_or_mul(s.bx[(size_t)jN * P + i] - s.bx[(size_t)j * P + i], c.dy, c.inv_dy);
    const T Jx = dBzdy, Jy = -dBzdx, Jz = dBydx - dBxdy;
    J2 = Jx * Jx + Jy * Jy + Jz * Jz;
    lap = (bzE - T(2) * bzC + bzW) * c.idx2 + (bzN - T(2) * bzC + bzS) * c.idy2;
}

template <class T>
__device__ __forceinline__ void joule_cell(const M2Const<T>& c, const Fields<T>& s, int i, int j, T dt,
                                           T& rho, T mx, T my, T mz, T& E, T& Bz, T Bx, T By) {
    if (!c.resistive) return;
    const T bzC = Bz;
    T J2, lap;
    joule_terms(c, s, i, j, bzC, J2, lap);
    E = E + dt * c.eta * J2;
    Bz = bzC + dt * c.eta * lap;
    floors(c, rho, mx, my, mz, E, Bx, By, Bz);
}

// ---------------------------------------------------------------------------
// Compensated (Kahan-style) accumulation of the conserved update, FP32 path.
// A compensated state stores every field as a pair (h, l): h the FP32 value
// the physics reads, l the rounding residual of h (|l| <= ulp(h)/2), so that
// h + l carries about twice FP32's digits between steps.  Every increment of
// a stage (flux divergence, CT, gravity kick, Joule heating and Bz diffusion)
// and the RK average are added with an error-free transformation (Knuth's
// TwoSum), which moves the rounding error of each addition into l instead of
// dropping it.  A floor that resets a value also resets its residual.
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ void comp_add(T& h, T& l, const T inc) {
    const T y = inc + l;
    const T s = h + y;
    const T bb = s - h;
    l = (h - (s - bb)) + (y - bb);
    h = s;
}

// (h, l) = 0.5 * ((ha + la) + (hb + lb)), compensated
template <class T>
__device__ __forceinline__ void comp_avg(const T ha, const T la, const T hb, const T lb, T& h, T& l) {
    const T s = ha + hb;
    const T bb = s - ha;
    T e = (ha - (s - bb)) + (hb - bb);
    e = e + (la + lb);
    const T r = s + e;            // fast two-sum: |s| >= |e|
    const T er = e - (r - s);
    h = T(0.5) * r;
    l = T(0.5) * er;
}

// enforce_floors on a compensated cell: a reset value starts a fresh residual
template <class T>
__device__ __forceinline__ void floors_comp(const M2Const<T>& c, T& rho, T& lrho, T mx, T my, T mz, T& E, T& lE,
                                            T Bx, T By, T Bz) {
    const T r0 = rho, e0 = E;
    floors(c, rho, mx, my, mz, E, Bx, By, Bz);
    if (rho != r0) lrho = T(0.0);
    if (E != e0) lE = T(0.0);
}

// joule_cell on a compensated cell: the increments of E and Bz go through comp_add
template <class T>
__device__ __forceinline__ void joule_cell_comp(const M2Const<T>& c, const Fields<T>& s, int i, int j, T dt,
                                                T& rho, T& lrho, T mx, T my, T mz, T& E, T& lE, T& Bz, T& lBz,
                                                T Bx, T By) {
    if (!c.resistive) return;
    T J2, lap;
    joule_terms(c, s, i, j, Bz, J2, lap);
    comp_add(E, lE, dt * c.eta * J2);
    comp_add(Bz, lBz, dt * c.eta * lap);
    floors_comp(c, rho, lrho, mx, my, mz, E, lE, Bx, By, Bz);
}

// ---------------------------------------------------------------------------
// One RK stage on one TX x TY tile whose first cell is (i0, j0).  DEFER: the
// input is a stored pre-Joule stage output whose Joule sub-step must be
// applied first.  GMODE selects the gravity source.  sm: StageGeomT::smem
// bytes of shared memory.  Called by the single-grid kernel (one tile per
// CTA) and by the batched persistent kernel (a run of tiles per CTA).
// ---------------------------------------------------------------------------
// REC: also store the updated cell state before its floors (rho, mx, my, mz,
// E, Bz into rec[0..5], pitched like the state): the record the discrete
// adjoint replays the floor and gravity-kick branches from.  NT_: threads of
// the CTA (at least TX * TY); SPLIT_ as in StageGeomT.
// KAHAN: compensated state (see comp_add): lin / lout hold the residuals of
// in / out; the tile's own cells read theirs and every increment is added
// with comp_add.  The physics (primitives, slopes, fluxes, EMFs) reads the
// FP32 values only, computed exactly as without KAHAN, so neighbouring tiles
// see identical primitives.  Needs kahan_smem_extra<T>(TX*TY) more bytes.
template <class T, int TX_, int TY_, bool DEFER, int GMODE, bool REC = false, int NT_ = TX_ * TY_,
          bool SPLIT_ = false, bool KAHAN = false>
__device__ __forceinline__ void m2_stage_tile(const M2Const<T>& c, const Fields<T>& in, const Fields<T>& out,
                                              const T* __restrict__ ga, const T* __restrict__ gb, const T dt,
                                              const int i0, const int j0, T* sm, T* const* rec = nullptr,
                                              const Fields<T> lin = Fields<T>{}, const Fields<T> lout = Fields<T>{}) {
    using G = StageGeomT<T, TX_, TY_, NT_, SPLIT_>;
    constexpr int TX = G::TX, TY = G::TY, HALO = G::HALO, RX = G::RX, RR = G::RR, NT = G::NT, NC = G::NC;
    constexpr int NFX = G::NFX, NGY = G::NGY, NSL = G::NSL;
    T* s_r = sm;          T* s_u = s_r + RR;   T* s_v = s_u + RR;   T* s_w = s_v + RR;
    T* s_P = s_w + RR;    T* s_bx = s_P + RR;  T* s_by = s_bx + RR; T* s_bz = s_by + RR;
    T* slx = s_bz + RR;         // 7 planes of NSL: slopes of cells (-1..TX) x (-1..TY), x direction
    T* sly = slx + 7 * (G::NSB - 1) * NSL;   // y direction (the same buffer, reused, unless SPLIT)
    T* fx = sly + 7 * NSL;      // 7 planes of NFX
    T* gy = fx + 7 * NFX;       // 7 planes of NGY
    T* ez = gy + 7 * NGY;       // NE
    T* own = ez + G::NE;        // 6 planes of NC
    T* own_lo = own + 6 * NC;   // KAHAN: 6 planes of NC, the residuals of own

    const int tid = threadIdx.x;
    const int P = c.pitch;

    // ---- A: primitives on the halo-2 region (get_prim_cc, M2:278-286) ----
    for (int k = tid; k < RR; k += NT) {
        const int rx = k % RX, ry = k / RX;
        const int gi = i0 - HALO + rx, gj = j0 - HALO + ry;
        const int ci = c.ax.cell(gi), cj = c.ay.cell(gj);
        const size_t q = (size_t)cj * P + ci;
        T rho = in.rho[q], mx = in.mx[q], my = in.my[q], mz = in.mz[q], E = in.E[q], Bz = in.Bz[q];
        const T Bx = T(0.5) * (in.bx[q] + in.bx[q + 1]);
        const T By = T(0.5) * (in.by[q] + in.by[q + P]);
        const int ox = rx - HALO, oy = ry - HALO;
        const bool mine = ox >= 0 && ox < TX && oy >= 0 && oy < TY;
        if constexpr (KAHAN) {
            if (mine) {   // the compensated pair of the tile's own cell, Joule sub-step included
                T h0 = rho, h4 = E, h5 = Bz;
                T l0 = lin.rho[q], l4 = lin.E[q], l5 = lin.Bz[q];
                if (DEFER) joule_cell_comp(c, in, ci, cj, dt, h0, l0, mx, my, mz, h4, l4, h5, l5, Bx, By);
                const int o = oy * TX + ox;
                own[o] = h0; own[NC + o] = mx; own[2 * NC + o] = my;
                own[3 * NC + o] = mz; own[4 * NC + o] = h4; own[5 * NC + o] = h5;
                own_lo[o] = l0; own_lo[NC + o] = lin.mx[q]; own_lo[2 * NC + o] = lin.my[q];
                own_lo[3 * NC + o] = lin.mz[q]; own_lo[4 * NC + o] = l4; own_lo[5 * NC + o] = l5;
            }
        }
        if (DEFER) joule_cell(c, in, ci, cj, dt, rho, mx, my, mz, E, Bz, Bx, By);
        const Prim<T> W = to_prim(c, rho, mx, my, mz, E, Bx, By, Bz);
        s_r[k] = W.r; s_u[k] = W.u; s_v[k] = W.v; s_w[k] = W.w;
        s_P[k] = W.P; s_bx[k] = W.bx; s_by[k] = W.by; s_bz[k] = W.bz;
        if (!KAHAN && mine) {
            const int o = oy * TX + ox;
            own[o] = rho; own[NC + o] = mx; own[2 * NC + o] = my;
            own[3 * NC + o] = mz; own[4 * NC + o] = E; own[5 * NC + o] = Bz;
        }
    }
    __syncthreads();

    // slope-buffer index of the cell at local (lx, ly), lx, ly in [-1, TX] x [-1, TY]
    auto sidx = [&](int lx, int ly) { return (ly + 1) * (TX + 2) + (lx + 1); };
    // region index of the same cell
    auto ridx = [&](int lx, int ly) { return (ly + HALO) * RX + (lx + HALO); };
    // MC slopes of one cell along stride st (recon_x / recon_y, M2:295-303, 319-327);
    // component 5 is the transverse in-plane B (By for x, Bx for y)
    auto slopes = [&](int k, int st, bool ydir, int o) {
        T* sl = ydir ? sly : slx;
        sl[o] = mc_slope(s_r[k - st], s_r[k], s_r[k + st]);
        sl[NSL + o] = mc_slope(s_u[k - st], s_u[k], s_u[k + st]);
        sl[2 * NSL + o] = mc_slope(s_v[k - st], s_v[k], s_v[k + st]);
        sl[3 * NSL + o] = mc_slope(s_w[k - st], s_w[k], s_w[k + st]);
        sl[4 * NSL + o] = mc_slope(s_P[k - st], s_P[k], s_P[k + st]);
        sl[5 * NSL + o] = ydir ? mc_slope(s_bx[k - st], s_bx[k], s_bx[k + st])
                               : mc_slope(s_by[k - st], s_by[k], s_by[k + st]);
        sl[6 * NSL + o] = mc_slope(s_bz[k - st], s_bz[k], s_bz[k + st]);
    };
    // face state of a cell: centre value + side * 0.5 * slope, then floors (M2:305-311)
    auto face_state = [&](int k, int o, bool ydir, T side) {
        const T* sl = ydir ? sly : slx;
        Prim<T> W;
        const T h = T(0.5) * side;
        W.r = s_r[k] + h * sl[o];
        W.u = s_u[k] + h * sl[NSL + o];
        W.v = s_v[k] + h * sl[2 * NSL + o];
        W.w = s_w[k] + h * sl[3 * NSL + o];
        W.P = s_P[k] + h * sl[4 * NSL + o];
        if (ydir) { W.bx = s_bx[k] + h * sl[5 * NSL + o]; W.by = s_by[k]; }
        else      { W.bx = s_bx[k]; W.by = s_by[k] + h * sl[5 * NSL + o]; }
        W.bz = s_bz[k] + h * sl[6 * NSL + o];
        W.r = vmax(W.r, c.floor_rho);
        W.P = vmax(W.P, c.floor_P);
        return W;
    };
    // FP32: the two face states of a face (cell kl's high side, cell kr's low
    // side) as packed pairs, already in hlld_x orientation (for a y face the
    // (u,v)/(Bx,By) swap of hlld_y; its Bx slot is set to Bn by hlld_x2)
    // (generic, so that only the FP32 instantiation forms it)
    auto face_pair = [&](auto kl, int ol, int kr, int orr, bool ydir) {
        const T* sl = ydir ? sly : slx;
        const float2 h = pk(0.5f, -0.5f);
        auto rec = [&](const T* v, int m) {
            return pfma(h, pk(sl[m * NSL + ol], sl[m * NSL + orr]), pk(v[kl], v[kr]));
        };
        auto ctr = [&](const T* v) { return pk(v[kl], v[kr]); };
        Prim2 S;
        S.r = rec(s_r, 0);
        S.P = rec(s_P, 4);
        S.w = rec(s_w, 3);
        S.bz = rec(s_bz, 6);
        if (ydir) {
            S.u = rec(s_v, 2); S.v = rec(s_u, 1); S.by = rec(s_bx, 5); S.bx = ctr(s_by);
        } else {
            S.u = rec(s_u, 1); S.v = rec(s_v, 2); S.by = rec(s_by, 5); S.bx = ctr(s_bx);
        }
        const float fr = (float)c.floor_rho, fp = (float)c.floor_P;
        S.r.x = fmaxf(S.r.x, fr); S.r.y = fmaxf(S.r.y, fr);
        S.P.x = fmaxf(S.P.x, fp); S.P.y = fmaxf(S.P.y, fp);
        return S;
    };

    auto x_slopes = [&](int k) {
        const int lx = k % (TX + 2) - 1, ly = k / (TX + 2) - 1;
        slopes(ridx(lx, ly), 1, false, k);
    };
    auto y_slopes = [&](int k) {
        const int lx = k % (TX + 2) - 1, ly = k / (TX + 2) - 1;
        slopes(ridx(lx, ly), RX, true, k);
    };
    // x faces i0..i0+TX, rows j0-1..j0+TY (M2:706-725)
    auto x_face = [&](int kk) {
        int f, r, k;
        if constexpr (G::ROW32) {   // kk = a lane of row r + 1
            f = kk % 32; r = kk / 32 - 1;
            if (f > TX) return;
            k = (r + 1) * (TX + 1) + f;
        } else {
            f = kk % (TX + 1); r = kk / (TX + 1) - 1; k = kk;
        }
        const int gi = i0 + f;
        if (gi > c.nx) return;
        const int cj = c.ay.cell(j0 + r);
        Flux<T> F;
        if constexpr (std::is_same<T, float>::value) {
            F = hlld_x2(c, face_pair(ridx(f - 1, r), sidx(f - 1, r), ridx(f, r), sidx(f, r), false),
                        in.bx[(size_t)cj * P + gi]);
        } else {
            const Prim<T> WL = face_state(ridx(f - 1, r), sidx(f - 1, r), false, T(1));
            const Prim<T> WR = face_state(ridx(f, r), sidx(f, r), false, T(-1));
            F = hlld_x(c, WL, WR, in.bx[(size_t)cj * P + gi]);
        }
        fx[k] = F.f0; fx[NFX + k] = F.f1; fx[2 * NFX + k] = F.f2; fx[3 * NFX + k] = F.f3;
        fx[4 * NFX + k] = F.f4; fx[5 * NFX + k] = F.f5; fx[6 * NFX + k] = F.f6;
    };
    // y faces j0..j0+TY, columns i0-1..i0+TX (M2:728-747)
    auto y_face = [&](int k) {
        const int col = k % (TX + 2) - 1, g = k / (TX + 2);
        const int gj = j0 + g;
        if (gj > c.ny) return;
        const int ci = c.ax.cell(i0 + col);
        Flux<T> Gf;
        if constexpr (std::is_same<T, float>::value) {
            Gf = hlld_x2(c, face_pair(ridx(col, g - 1), sidx(col, g - 1), ridx(col, g), sidx(col, g), true),
                         in.by[(size_t)gj * P + ci]);
            const T t = Gf.f1; Gf.f1 = Gf.f2; Gf.f2 = t;   // hlld_y's swap back
        } else {
            const Prim<T> WL = face_state(ridx(col, g - 1), sidx(col, g - 1), true, T(1));
            const Prim<T> WR = face_state(ridx(col, g), sidx(col, g), true, T(-1));
            Gf = hlld_y(c, WL, WR, in.by[(size_t)gj * P + ci]);
        }
        gy[k] = Gf.f0; gy[NGY + k] = Gf.f1; gy[2 * NGY + k] = Gf.f2; gy[3 * NGY + k] = Gf.f3;
        gy[4 * NGY + k] = Gf.f4; gy[5 * NGY + k] = Gf.f5; gy[6 * NGY + k] = Gf.f6;
    };
    if constexpr (G::SPLIT) {
        // ---- B: x and y slopes; C: x and y face fluxes (ranges padded to whole warps) ----
        constexpr int NSLP = (NSL + 31) / 32 * 32, NFXP = (NFX + 31) / 32 * 32;
        for (int k = tid; k < NSLP + NSL; k += NT) {
            if (k < NSL) x_slopes(k);
            else if (k >= NSLP) y_slopes(k - NSLP);
        }
        __syncthreads();
        for (int k = tid; k < NFXP + NGY; k += NT) {
            if (k < NFX) x_face(k);
            else if (k >= NFXP) y_face(k - NFXP);
        }
        __syncthreads();
    } else {
        // ---- B: x slopes, then x faces; C: y slopes (same buffer), then y faces ----
        for (int k = tid; k < NSL; k += NT) x_slopes(k);
        if constexpr (G::ROWSYNC) __syncwarp(); else __syncthreads();
        for (int k = tid; k < (G::ROW32 ? 32 * (TY + 2) : NFX); k += NT) x_face(k);
        if constexpr (G::ROWSYNC) __syncwarp(); else __syncthreads();
        for (int k = tid; k < NSL; k += NT) y_slopes(k);
        __syncthreads();
        for (int k = tid; k < NGY; k += NT) y_face(k);
        // ROWSYNC: warp w computes y-face row w and then edge row w, which reads
        // that y-face row and the x faces (written before the last barrier)
        if constexpr (G::ROWSYNC) __syncwarp(); else __syncthreads();
    }

    // ---- E: edge EMFs, edges i0..i0+TX x j0..j0+TY (M2:782-804, 565-575) ----
    for (int kk = tid; kk < (G::ROW32 ? 32 * (TY + 1) : G::NE); kk += NT) {
        const int ei = G::ROW32 ? kk % 32 : kk % (TX + 1), ej = G::ROW32 ? kk / 32 : kk / (TX + 1);
        if (G::ROW32 && ei > TX) continue;
        const int k = ej * (TX + 1) + ei;
        const int ie = i0 + ei, je = j0 + ej;
        if (ie > c.nx || je > c.ny) continue;
        const T exm = -fx[5 * NFX + ej * (TX + 1) + ei];        // x face ie, row je-1
        const T ex0 = -fx[5 * NFX + (ej + 1) * (TX + 1) + ei];  // x face ie, row je
        const T eym = gy[5 * NGY + ej * (TX + 2) + ei];         // y face je, col ie-1
        const T ey0 = gy[5 * NGY + ej * (TX + 2) + ei + 1];     // y face je, col ie
        const T ideal = T(0.25) * (exm + ex0 + eym + ey0);
        T res = T(0.0);
        if (c.resistive) {
            const int ci = c.ax.cell(ie), cim = c.ax.cell(ie - 1);
            const int cj = c.ay.cell(je), cjm = c.ay.cell(je - 1);
            const T dBydx = div_or_mul(in.by[(size_t)je * P + ci] - in.by[(size_t)je * P + cim], c.dx, c.inv_dx);
            const T dBxdy = div_or_mul(in.bx[(size_t)cj * P + ie] - in.bx[(size_t)cjm * P + ie], c.dy, c.inv_dy);
            res = c.eta * (dBydx - dBxdy);
        }
        ez[k] = ideal + res;
    }
    __syncthreads();

    // ---- D+F: FV update, floors, CT, gravity kick, store (M2:750-779, 807-832) ----
    const int tx = G::ROW32 ? tid % 32 : tid % TX, ty = G::ROW32 ? tid / 32 : tid / TX;
    if (tx >= TX || ty >= TY) return;
    const int gi = i0 + tx, gj = j0 + ty;
    if (gi >= c.nx || gj >= c.ny) return;
    const size_t q = (size_t)gj * P + gi;
    const int o = ty * TX + tx;
    T rho = own[o], mx = own[NC + o], my = own[2 * NC + o];
    T mz = own[3 * NC + o], E = own[4 * NC + o], Bz = own[5 * NC + o];
    T lrho = T(0.0), lmx = T(0.0), lmy = T(0.0), lmz = T(0.0), lE = T(0.0), lBz = T(0.0);
    if constexpr (KAHAN) {
        lrho = own_lo[o]; lmx = own_lo[NC + o]; lmy = own_lo[2 * NC + o];
        lmz = own_lo[3 * NC + o]; lE = own_lo[4 * NC + o]; lBz = own_lo[5 * NC + o];
    }
    {
        const int kxL = (ty + 1) * (TX + 1) + tx;
        const int kgD = ty * (TX + 2) + tx + 1, kgU = kgD + (TX + 2);
        T d[7];
#pragma unroll
        for (int m = 0; m < 7; m++)
            d[m] = -(fx[m * NFX + kxL + 1] - fx[m * NFX + kxL]) * c.inv_dx -
                   (gy[m * NGY + kgU] - gy[m * NGY + kgD]) * c.inv_dy;
        const int kc = ridx(tx, ty);
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
            if (REC) {
                rec[0][q] = rho; rec[1][q] = mx; rec[2][q] = my; rec[3][q] = mz; rec[4][q] = E; rec[5][q] = Bz;
            }
            floors(c, rho, mx, my, mz, E, s_bx[kc], s_by[kc], Bz);
        }
    }
    // CT (M2:807-830) for this cell's four faces
    const T dtdy = dt / c.dy, dtdx = dt / c.dx;
    const T e00 = ez[ty * (TX + 1) + tx], e10 = ez[ty * (TX + 1) + tx + 1];
    const T e01 = ez[(ty + 1) * (TX + 1) + tx], e11 = ez[(ty + 1) * (TX + 1) + tx + 1];
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

    // gravity kick + floors with the post-CT B (add_gravity_sources, M2:602-629)
    if (GMODE != GRAV_NONE && c.gravity_on) {
        T gxq, gyq;
        if (GMODE == GRAV_ARRAYS) {
            gxq = ga[q]; gyq = gb[q];
        } else {
            const T* phi = ga;
            const int iE = c.ax.cell(gi + 1), iW = c.ax.cell(gi - 1);
            const int jN = c.ay.cell(gj + 1), jS = c.ay.cell(gj - 1);
            gxq = div_or_mul(-(phi[(size_t)gj * P + iE] - phi[(size_t)gj * P + iW]), c.two_dx, T(0.5) * c.inv_dx);
            gyq = div_or_mul(-(phi[(size_t)jN * P + gi] - phi[(size_t)jS * P + gi]), c.two_dy, T(0.5) * c.inv_dy);
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
        lout.rho[q] = lrho; lout.mx[q] = lmx; lout.my[q] = lmy; lout.mz[q] = lmz; lout.E[q] = lE; lout.Bz[q] = lBz;
    }
}

// extra shared memory of a KAHAN stage tile of nc cells (the residuals of its own cells)
template <class T> constexpr size_t kahan_smem_extra(int nc) { return sizeof(T) * 6 * (size_t)nc; }

template <class T, bool DEFER, int GMODE>
__global__ void __launch_bounds__(StageGeom<T>::NT, StageTile<T>::MINB)
m2_stage_kernel(const M2Const<T> c, const Fields<T> in, const Fields<T> out, const T* __restrict__ ga,
                const T* __restrict__ gb, const double* __restrict__ dtp, const int* __restrict__ active) {
    constexpr int TX = StageTile<T>::TX, TY = StageTile<T>::TY;
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    m2_stage_tile<T, TX, TY, DEFER, GMODE, false, StageTile<T>::NT, StageTile<T>::SPLIT>(
        c, in, out, ga, gb, (T)(*dtp), blockIdx.x * TX, blockIdx.y * TY, reinterpret_cast<T*>(smem_raw));
}

// the same stage on a compensated state (lin / lout: residuals of in / out)
template <class T, bool DEFER, int GMODE>
__global__ void __launch_bounds__(StageGeom<T>::NT, StageTile<T>::MINB)
m2_stage_comp_kernel(const M2Const<T> c, const Fields<T> in, const Fields<T> out, const Fields<T> lin,
                     const Fields<T> lout, const T* __restrict__ ga, const T* __restrict__ gb,
                     const double* __restrict__ dtp, const int* __restrict__ active) {
    constexpr int TX = StageTile<T>::TX, TY = StageTile<T>::TY;
    if (active && *active == 0) return;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    m2_stage_tile<T, TX, TY, DEFER, GMODE, false, StageTile<T>::NT, StageTile<T>::SPLIT, true>(
        c, in, out, ga, gb, (T)(*dtp), blockIdx.x * TX, blockIdx.y * TY, reinterpret_cast<T*>(smem_raw), nullptr,
        lin, lout);
}

// ---------------------------------------------------------------------------
// RK average (M2:848-868) of one cell, fused with the deferred stage-2 Joule
// sub-step; returns the CFL speed of the result (compute_dt's loop body,
// M2:585-587) and adds its density to rsum.  Inactive (t >= t_end): U^n is
// carried over unchanged so that the buffer rotation stays valid.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ double average_cell(const M2Const<T>& c, const Fields<T>& un, const Fields<T>& s2,
                                               const Fields<T>& out, const T dt, const bool act, const int i,
                                               const int j, double& rsum) {
    const int P = c.pitch;
    const size_t q = (size_t)j * P + i;
    if (!act) {
        const T rho = un.rho[q], mx = un.mx[q], my = un.my[q], mz = un.mz[q], E = un.E[q], Bz = un.Bz[q];
        const T bxl = un.bx[q], bxr = un.bx[q + 1], byd = un.by[q], byu = un.by[q + P];
        out.rho[q] = rho; out.mx[q] = mx; out.my[q] = my; out.mz[q] = mz; out.E[q] = E; out.Bz[q] = Bz;
        out.bx[q] = bxl;
        if (i == c.nx - 1) out.bx[q + 1] = bxr;
        out.by[q] = byd;
        if (j == c.ny - 1) out.by[q + P] = byu;
        const Prim<T> W = to_prim(c, rho, mx, my, mz, E, T(0.5) * (bxl + bxr), T(0.5) * (byd + byu), Bz);
        rsum += (double)rho;
        return (double)vmax(fabs(W.u) + fast_speed(c, W, W.bx), fabs(W.v) + fast_speed(c, W, W.by));
    }
    T rho = s2.rho[q], mx = s2.mx[q], my = s2.my[q], mz = s2.mz[q], E = s2.E[q], Bz = s2.Bz[q];
    const T bxl2 = s2.bx[q], bxr2 = s2.bx[q + 1], byd2 = s2.by[q], byu2 = s2.by[q + P];
    joule_cell(c, s2, i, j, dt, rho, mx, my, mz, E, Bz, T(0.5) * (bxl2 + bxr2), T(0.5) * (byd2 + byu2));
    rho = T(0.5) * (un.rho[q] + rho);
    mx = T(0.5) * (un.mx[q] + mx);
    my = T(0.5) * (un.my[q] + my);
    mz = T(0.5) * (un.mz[q] + mz);
    E = T(0.5) * (un.E[q] + E);
    Bz = T(0.5) * (un.Bz[q] + Bz);
    const T bxl = T(0.5) * (un.bx[q] + bxl2), bxr = T(0.5) * (un.bx[q + 1] + bxr2);
    const T byd = T(0.5) * (un.by[q] + byd2), byu = T(0.5) * (un.by[q + P] + byu2);
    const T Bx = T(0.5) * (bxl + bxr), By = T(0.5) * (byd + byu);
    floors(c, rho, mx, my, mz, E, Bx, By, Bz);
    out.rho[q] = rho; out.mx[q] = mx; out.my[q] = my; out.mz[q] = mz; out.E[q] = E; out.Bz[q] = Bz;
    out.bx[q] = bxl;
    if (i == c.nx - 1) out.bx[q + 1] = bxr;
    out.by[q] = byd;
    if (j == c.ny - 1) out.by[q + P] = byu;
    const Prim<T> W = to_prim(c, rho, mx, my, mz, E, Bx, By, Bz);
    const T sx = fabs(W.u) + fast_speed(c, W, W.bx);
    const T sy = fabs(W.v) + fast_speed(c, W, W.by);
    rsum += (double)rho;
    return (double)vmax(sx, sy);
}

// average_cell on compensated states: unl, s2l, outl hold the residuals of
// un, s2, out.  The Joule increments of stage 2 and the average go through
// comp_add / comp_avg; floors reset the residual of a value they reset.
template <class T>
__device__ __forceinline__ double average_cell_comp(const M2Const<T>& c, const Fields<T>& un, const Fields<T>& s2,
                                                    const Fields<T>& out, const Fields<T>& unl,
                                                    const Fields<T>& s2l, const Fields<T>& outl, const T dt,
                                                    const bool act, const int i, const int j, double& rsum) {
    const int P = c.pitch;
    const size_t q = (size_t)j * P + i;
    if (!act) {
        T* dst[8] = {out.rho, out.mx, out.my, out.mz, out.E, out.Bz, out.bx, out.by};
        T* dstl[8] = {outl.rho, outl.mx, outl.my, outl.mz, outl.E, outl.Bz, outl.bx, outl.by};
        const T* src[8] = {un.rho, un.mx, un.my, un.mz, un.E, un.Bz, un.bx, un.by};
        const T* srcl[8] = {unl.rho, unl.mx, unl.my, unl.mz, unl.E, unl.Bz, unl.bx, unl.by};
#pragma unroll
        for (int m = 0; m < 8; m++) { dst[m][q] = src[m][q]; dstl[m][q] = srcl[m][q]; }
        if (i == c.nx - 1) { out.bx[q + 1] = un.bx[q + 1]; outl.bx[q + 1] = unl.bx[q + 1]; }
        if (j == c.ny - 1) { out.by[q + P] = un.by[q + P]; outl.by[q + P] = unl.by[q + P]; }
        const T bxl = un.bx[q], bxr = un.bx[q + 1], byd = un.by[q], byu = un.by[q + P];
        const Prim<T> W = to_prim(c, un.rho[q], un.mx[q], un.my[q], un.mz[q], un.E[q], T(0.5) * (bxl + bxr),
                                  T(0.5) * (byd + byu), un.Bz[q]);
        rsum += (double)un.rho[q];
        return (double)vmax(fabs(W.u) + fast_speed(c, W, W.bx), fabs(W.v) + fast_speed(c, W, W.by));
    }
    T rho = s2.rho[q], mx = s2.mx[q], my = s2.my[q], mz = s2.mz[q], E = s2.E[q], Bz = s2.Bz[q];
    T lrho = s2l.rho[q], lmx = s2l.mx[q], lmy = s2l.my[q], lmz = s2l.mz[q], lE = s2l.E[q], lBz = s2l.Bz[q];
    const T bxl2 = s2.bx[q], bxr2 = s2.bx[q + 1], byd2 = s2.by[q], byu2 = s2.by[q + P];
    joule_cell_comp(c, s2, i, j, dt, rho, lrho, mx, my, mz, E, lE, Bz, lBz, T(0.5) * (bxl2 + bxr2),
                    T(0.5) * (byd2 + byu2));
    comp_avg(un.rho[q], unl.rho[q], rho, lrho, rho, lrho);
    comp_avg(un.mx[q], unl.mx[q], mx, lmx, mx, lmx);
    comp_avg(un.my[q], unl.my[q], my, lmy, my, lmy);
    comp_avg(un.mz[q], unl.mz[q], mz, lmz, mz, lmz);
    comp_avg(un.E[q], unl.E[q], E, lE, E, lE);
    comp_avg(un.Bz[q], unl.Bz[q], Bz, lBz, Bz, lBz);
    T bxl, bxr, byd, byu, lbxl, lbxr, lbyd, lbyu;
    comp_avg(un.bx[q], unl.bx[q], bxl2, s2l.bx[q], bxl, lbxl);
    comp_avg(un.bx[q + 1], unl.bx[q + 1], bxr2, s2l.bx[q + 1], bxr, lbxr);
    comp_avg(un.by[q], unl.by[q], byd2, s2l.by[q], byd, lbyd);
    comp_avg(un.by[q + P], unl.by[q + P], byu2, s2l.by[q + P], byu, lbyu);
    const T Bx = T(0.5) * (bxl + bxr), By = T(0.5) * (byd + byu);
    floors_comp(c, rho, lrho, mx, my, mz, E, lE, Bx, By, Bz);
    out.rho[q] = rho; out.mx[q] = mx; out.my[q] = my; out.mz[q] = mz; out.E[q] = E; out.Bz[q] = Bz;
    outl.rho[q] = lrho; outl.mx[q] = lmx; outl.my[q] = lmy; outl.mz[q] = lmz; outl.E[q] = lE; outl.Bz[q] = lBz;
    out.bx[q] = bxl; outl.bx[q] = lbxl;
    if (i == c.nx - 1) { out.bx[q + 1] = bxr; outl.bx[q + 1] = lbxr; }
    out.by[q] = byd; outl.by[q] = lbyd;
    if (j == c.ny - 1) { out.by[q + P] = byu; outl.by[q + P] = lbyu; }
    const Prim<T> W = to_prim(c, rho, mx, my, mz, E, Bx, By, Bz);
    const T sx = fabs(W.u) + fast_speed(c, W, W.bx);
    const T sy = fabs(W.v) + fast_speed(c, W, W.by);
    rsum += (double)rho;
    return (double)vmax(sx, sy);
}

// CFL speed of one cell of a state (compute_dt's loop body, M2:585-587)
template <class T>
__device__ __forceinline__ double speed_cell(const M2Const<T>& c, const Fields<T>& s, const int i, const int j) {
    const size_t q = (size_t)j * c.pitch + i;
    const T Bx = T(0.5) * (s.bx[q] + s.bx[q + 1]), By = T(0.5) * (s.by[q] + s.by[q + c.pitch]);
    const Prim<T> W = to_prim(c, s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], Bx, By, s.Bz[q]);
    const T sx = fabs(W.u) + fast_speed(c, W, W.bx);
    const T sy = fabs(W.v) + fast_speed(c, W, W.by);
    return (double)vmax(sx, sy);
}

// RK average over the whole grid; emits the CFL and density partials of
// U^{n+1} for the next step.  un: U^n, s2: stage-2 output (pre-Joule), out: U^{n+1}.
template <class T, int NT>
__global__ void __launch_bounds__(NT)
m2_average_kernel(const M2Const<T> c, const Fields<T> un, const Fields<T> s2, const Fields<T> out,
                  const double* __restrict__ dtp, const int* __restrict__ active, double* __restrict__ spd_part,
                  double* __restrict__ rho_part) {
    const bool act = (active == nullptr) || (*active != 0);
    __shared__ double sh[NT / 32];
    const T dt = (T)(*dtp);
    double smax = 0.0, rsum = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const double s = average_cell(c, un, s2, out, dt, act, k % c.nx, k / c.nx, rsum);
        if (s > smax) smax = s;   // NaN never wins, as in std::max(maxs, x)
    }
    const double bm = block_max<NT>(smax, sh);
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) { spd_part[blockIdx.x] = bm; rho_part[blockIdx.x] = bs; }
}

// m2_average_kernel on compensated states
template <class T, int NT>
__global__ void __launch_bounds__(NT)
m2_average_comp_kernel(const M2Const<T> c, const Fields<T> un, const Fields<T> s2, const Fields<T> out,
                       const Fields<T> unl, const Fields<T> s2l, const Fields<T> outl,
                       const double* __restrict__ dtp, const int* __restrict__ active,
                       double* __restrict__ spd_part, double* __restrict__ rho_part) {
    const bool act = (active == nullptr) || (*active != 0);
    __shared__ double sh[NT / 32];
    const T dt = (T)(*dtp);
    double smax = 0.0, rsum = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const double s = average_cell_comp(c, un, s2, out, unl, s2l, outl, dt, act, k % c.nx, k / c.nx, rsum);
        if (s > smax) smax = s;
    }
    const double bm = block_max<NT>(smax, sh);
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) { spd_part[blockIdx.x] = bm; rho_part[blockIdx.x] = bs; }
}

// CFL speed reduction and density sum of a state (compute_dt, M2:579-598).
template <class T, int NT>
__global__ void __launch_bounds__(NT)
m2_speed_kernel(const M2Const<T> c, const Fields<T> s, double* __restrict__ spd_part, double* __restrict__ rho_part) {
    __shared__ double sh[NT / 32];
    const int P = c.pitch;
    double smax = 0.0, rsum = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const int i = k % c.nx, j = k / c.nx;
        const double v = speed_cell(c, s, i, j);
        if (v > smax) smax = v;
        rsum += (double)s.rho[(size_t)j * P + i];
    }
    const double bm = block_max<NT>(smax, sh);
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) { spd_part[blockIdx.x] = bm; rho_part[blockIdx.x] = bs; }
}

// Sum of the density of a state (for the Poisson mean).
template <class T, int NT>
__global__ void __launch_bounds__(NT)
m2_rho_sum_kernel(const M2Const<T> c, const T* __restrict__ rho, double* __restrict__ rho_part) {
    __shared__ double sh[NT / 32];
    double rsum = 0.0;
    const int ncell = c.nx * c.ny;
#pragma unroll 8
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {   // loads issued ahead, sum in order
        const int i = k % c.nx, j = k / c.nx;
        rsum += (double)rho[(size_t)j * c.pitch + i];
    }
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) rho_part[blockIdx.x] = bs;
}

// Host-visible diagnostics of a state: FP64 sums and max |div B| (M2:873-879).
template <class T, int NT>
__global__ void __launch_bounds__(NT)
m2_diag_kernel(const M2Const<T> c, const Fields<T> s, double* __restrict__ part /* 7 * gridDim.x */) {
    __shared__ double sh[NT / 32];
    const int P = c.pitch;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    double dmax = 0.0;
    double nonfinite = 0.0;
    const int ncell = c.nx * c.ny;
    for (int k = blockIdx.x * NT + threadIdx.x; k < ncell; k += gridDim.x * NT) {
        const int i = k % c.nx, j = k / c.nx;
        const size_t q = (size_t)j * P + i;
        const double v[6] = {(double)s.rho[q], (double)s.mx[q], (double)s.my[q], (double)s.mz[q], (double)s.E[q],
                             (double)s.Bz[q]};
        for (int m = 0; m < 6; m++) {
            acc[m] += v[m];
            if (!isfinite(v[m])) nonfinite = 1.0;
        }
        // divB_cc with the reference's face lookups (i+1, j+1 never wrap for a cell)
        const double d = ((double)s.bx[q + 1] - (double)s.bx[q]) / (double)c.dx +
                         ((double)s.by[q + P] - (double)s.by[q]) / (double)c.dy;
        dmax = fmax(dmax, fabs(d));
    }
    for (int m = 0; m < 5; m++) {
        const double b = block_sum<NT>(acc[m], sh);
        if (threadIdx.x == 0) part[m * gridDim.x + blockIdx.x] = b;
    }
    const double bm = block_max<NT>(dmax, sh);
    const double bn = block_max<NT>(nonfinite, sh);
    if (threadIdx.x == 0) { part[5 * gridDim.x + blockIdx.x] = bm; part[6 * gridDim.x + blockIdx.x] = bn; }
}

// Derived snapshot fields of the reference main()'s store (M2:1065-1106), in
// its output order: rho, P, Mach, u, v, vabs, Bx, By, Bz (cell-centred, from
// the faces) and div B; out holds 10 planes of nx*ny doubles, row-major.
// Primitives through cons_to_prim, cs = sqrt(max(0, gamma P / max(rho,
// floor_rho))), Mach = |v| / max(cs, 1e-14); in the state precision, the
// divergence in FP64 as in the diagnostics.
template <class T>
__global__ void m2_derived_kernel(const M2Const<T> c, const Fields<T> s, double* __restrict__ out) {
    const int P = c.pitch;
    const size_t n = (size_t)c.nx * c.ny;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k % c.nx), j = (int)(k / c.nx);
        const size_t q = (size_t)j * P + i;
        const T Bx = T(0.5) * (s.bx[q] + s.bx[q + 1]);
        const T By = T(0.5) * (s.by[q] + s.by[q + P]);
        const Prim<T> W = to_prim(c, s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], Bx, By, s.Bz[q]);
        const T cs = sqrt(vmax(T(0.0), c.gamma * W.P / vmax(W.r, c.floor_rho)));
        const T vabs = sqrt(W.u * W.u + W.v * W.v + W.w * W.w);
        const T mach = vabs / vmax(cs, T(1e-14));
        const double div = ((double)s.bx[q + 1] - (double)s.bx[q]) / (double)c.dx +
                           ((double)s.by[q + P] - (double)s.by[q]) / (double)c.dy;
        out[k] = W.r;
        out[n + k] = W.P;
        out[2 * n + k] = mach;
        out[3 * n + k] = W.u;
        out[4 * n + k] = W.v;
        out[5 * n + k] = vabs;
        out[6 * n + k] = Bx;
        out[7 * n + k] = By;
        out[8 * n + k] = W.bz;
        out[9 * n + k] = div;
    }
}

// Combine CFL partials into dt (M2:590-597), clamp to t_end (M2:1114) and set
// the active flag that makes the step kernels no-ops once t >= t_end.
struct DtSpec {
    double cfl, hmin, eta, t_end;
    int clamp_to_end;
    double seed;      // initial value of the speed maximum (M2/M3: 1e-14, EH: 1e-30)
    double end_eps;   // loop runs while t < t_end - end_eps (M2/M3: 0, EH: 1e-14)
    int check;        // 1: flag a non-finite or non-positive dt (EH:699-702)
    int cap;          // 1: dt = min(dt_h, dt_r), dt_r = 1e100 or the resistive limit (M2:592-597, M3:643-647)
};

// Host <-> device layout conversion: contiguous FP64 reference layout with row
// length w and h rows  <->  pitched T field.
// rows over blockIdx.y, columns over blockIdx.x (no index division)
template <class T>
__global__ void pack_in_kernel(const double* __restrict__ src, T* __restrict__ dst, int w, int h, int pitch) {
    for (int j = blockIdx.y; j < h; j += gridDim.y)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w; i += gridDim.x * blockDim.x)
            dst[(size_t)j * pitch + i] = (T)src[(size_t)j * w + i];
}
template <class T>
__global__ void pack_out_kernel(const T* __restrict__ src, double* __restrict__ dst, int w, int h, int pitch) {
    for (int j = blockIdx.y; j < h; j += gridDim.y)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w; i += gridDim.x * blockDim.x)
            dst[(size_t)j * w + i] = (double)src[(size_t)j * pitch + i];
}
// compensated state: hi = the FP64 value rounded to T, lo = the rounding residual (in T)
template <class T>
__global__ void pack_in_split_kernel(const double* __restrict__ src, T* __restrict__ hi, T* __restrict__ lo, int w,
                                     int h, int pitch) {
    for (int j = blockIdx.y; j < h; j += gridDim.y)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w; i += gridDim.x * blockDim.x) {
            const double v = src[(size_t)j * w + i];
            const T a = (T)v;
            hi[(size_t)j * pitch + i] = a;
            lo[(size_t)j * pitch + i] = (T)(v - (double)a);
        }
}
// compensated state -> FP64: hi + lo (exact in FP64 for FP32 pairs)
template <class T>
__global__ void pack_out_sum_kernel(const T* __restrict__ hi, const T* __restrict__ lo, double* __restrict__ dst,
                                    int w, int h, int pitch) {
    for (int j = blockIdx.y; j < h; j += gridDim.y)
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < w; i += gridDim.x * blockDim.x)
            dst[(size_t)j * w + i] = (double)hi[(size_t)j * pitch + i] + (double)lo[(size_t)j * pitch + i];
}

}  // namespace ccb
