// 3D resistive-MHD step kernels (mhd3d_resistive_hlld_ct.cpp, cited M3:<line>),
// templated on T; instantiated per precision in mhd3d_f64.cu / mhd3d_f32.cu.
//
// Layout: every field is a pitched 3D array, element (i,j,k) at
// k*PS + j*P + i with P = round_up(Nx+1, 32), PS = P*(Ny+1) and Nz+1 planes, so
// cells, the three face arrays (index N along their own axis), the edge
// arrays and the face-flux arrays all share one indexing.
//
// One RK stage (advance_stage, M3:694-1030) is a short pipeline of kernels
// addressed by actual cell / face / edge indices with the reference's own wrap
// rules (cells mod N or clamp; faces mod N+1 or clamp; cell-centred B formed
// from unwrapped indices through the face lookups, as M3:280-296 do):
//   m3_prim_kernel    primitives of every cell (stage 2: first the deferred
//                     Joule heating + floors of stage 1, in place)
//   m3_face_kernel    MUSCL-MC face states + HLLD for x, y or z faces;
//                     5 flux components and the two face EMFs per face
//   m3_update_kernel  FV update + floors with the stage-input B
//   m3_emf_ct_kernel  edge EMFs (average of four face EMFs + eta J from
//                     cell-centred B) and the CT update of the three face
//                     arrays, the EMFs kept on chip
// The Joule sub-step (M3:1017) needs the post-CT faces of neighbouring cells,
// so it is applied by the next kernel that reads the stage output (the stage-2
// prim kernel, the RK average).  It changes only E of its own cell, so doing it
// in place is race-free.
#pragma once
#include "mhd3d_physics.cuh"

namespace ccb {

template <class T> struct Fields3 {
    T* rho; T* mx; T* my; T* mz; T* E; T* bx; T* by; T* bz;
};

// per-direction face data: 5 flux components + 2 face EMFs, each a full plane set
template <class T> struct FaceData {
    T* f[7];
};

// ---- face and cell-centred B with the reference's index rules (M3:250-296) ----
template <class T>
__device__ __forceinline__ T bxf3(const M3Const<T>& c, const T* bx, int i, int j, int k) {
    return bx[c.idx(c.ax.face(i), c.ay.cell(j), c.az.cell(k))];
}
template <class T>
__device__ __forceinline__ T byf3(const M3Const<T>& c, const T* by, int i, int j, int k) {
    return by[c.idx(c.ax.cell(i), c.ay.face(j), c.az.cell(k))];
}
template <class T>
__device__ __forceinline__ T bzf3(const M3Const<T>& c, const T* bz, int i, int j, int k) {
    return bz[c.idx(c.ax.cell(i), c.ay.cell(j), c.az.face(k))];
}
template <class T>
__device__ __forceinline__ T bx_cc3(const M3Const<T>& c, const T* bx, int i, int j, int k) {
    return T(0.5) * (bxf3(c, bx, i, j, k) + bxf3(c, bx, i + 1, j, k));
}
template <class T>
__device__ __forceinline__ T by_cc3(const M3Const<T>& c, const T* by, int i, int j, int k) {
    return T(0.5) * (byf3(c, by, i, j, k) + byf3(c, by, i, j + 1, k));
}
template <class T>
__device__ __forceinline__ T bz_cc3(const M3Const<T>& c, const T* bz, int i, int j, int k) {
    return T(0.5) * (bzf3(c, bz, i, j, k) + bzf3(c, bz, i, j, k + 1));
}

// Joule heating E += dt eta |J|^2 of cell (i,j,k) (add_joule_heating, M3:652-692)
template <class T>
__device__ __forceinline__ T joule3(const M3Const<T>& c, const Fields3<T>& s, int i, int j, int k, T dt) {
    const T dBzdy = (bz_cc3(c, s.bz, i, j + 1, k) - bz_cc3(c, s.bz, i, j - 1, k)) / c.two_dy;
    const T dBydz = (by_cc3(c, s.by, i, j, k + 1) - by_cc3(c, s.by, i, j, k - 1)) / c.two_dz;
    const T dBxdz = (bx_cc3(c, s.bx, i, j, k + 1) - bx_cc3(c, s.bx, i, j, k - 1)) / c.two_dz;
    const T dBzdx = (bz_cc3(c, s.bz, i + 1, j, k) - bz_cc3(c, s.bz, i - 1, j, k)) / c.two_dx;
    const T dBydx = (by_cc3(c, s.by, i + 1, j, k) - by_cc3(c, s.by, i - 1, j, k)) / c.two_dx;
    const T dBxdy = (bx_cc3(c, s.bx, i, j + 1, k) - bx_cc3(c, s.bx, i, j - 1, k)) / c.two_dy;
    const T Jx = dBzdy - dBydz, Jy = dBxdz - dBzdx, Jz = dBydx - dBxdy;
    const T J2 = Jx * Jx + Jy * Jy + Jz * Jz;
    return dt * c.eta * J2;
}

// Cell-centred B planes of a state (bx_cc3, by_cc3, bz_cc3 of every cell),
// written once before a Joule pass so that the pass reads 12 stored values per
// cell instead of forming them from 24 face loads.  The values are the same
// doubles: bx_cc3(i, j, k) of a neighbour (i', j', k') outside the box equals
// the stored value at its mapped cell, the cell map being idempotent.
template <class T> struct Bcc3 { T* x; T* y; T* z; };

// Joule heating of cell (i,j,k) in the box (add_joule_heating, M3:652-692),
// as joule3 with the cell-centred B read from b
template <class T>
__device__ __forceinline__ T joule3_cc(const M3Const<T>& c, const Bcc3<T>& b, int i, int j, int k, T dt) {
    auto at = [&](const T* f, int a, int bb, int d) { return f[c.idx(a, bb, d)]; };
    const int ip = c.ax.cell(i + 1), im = c.ax.cell(i - 1), jp = c.ay.cell(j + 1), jm = c.ay.cell(j - 1);
    const int kp = c.az.cell(k + 1), km = c.az.cell(k - 1);
    const T dBzdy = (at(b.z, i, jp, k) - at(b.z, i, jm, k)) / c.two_dy;
    const T dBydz = (at(b.y, i, j, kp) - at(b.y, i, j, km)) / c.two_dz;
    const T dBxdz = (at(b.x, i, j, kp) - at(b.x, i, j, km)) / c.two_dz;
    const T dBzdx = (at(b.z, ip, j, k) - at(b.z, im, j, k)) / c.two_dx;
    const T dBydx = (at(b.y, ip, j, k) - at(b.y, im, j, k)) / c.two_dx;
    const T dBxdy = (at(b.x, i, jp, k) - at(b.x, i, jm, k)) / c.two_dy;
    const T Jx = dBzdy - dBydz, Jy = dBxdz - dBzdx, Jz = dBydx - dBxdy;
    const T J2 = Jx * Jx + Jy * Jy + Jz * Jz;
    return dt * c.eta * J2;
}

// grid-stride helper over an (nx, ny, nz) box with 32-bit indices (the handle
// rejects grids whose (Nx+1)(Ny+1)(Nz+1) reaches 2^31)
#define CC_FOR3(nx_, ny_, nz_)                                                                          \
    const unsigned w3_ = (unsigned)(nx_), h3_ = (unsigned)(ny_);                                        \
    const unsigned n3_ = w3_ * h3_ * (unsigned)(nz_);                                                   \
    for (unsigned t_ = blockIdx.x * blockDim.x + threadIdx.x; t_ < n3_; t_ += gridDim.x * blockDim.x)
// the (i, j, k) of t_ inside CC_FOR3, two 32-bit divisions
#define CC_IJK3(i, j, k)                                                                                \
    const unsigned r3_ = t_ / w3_, q3_ = r3_ / h3_;                                                     \
    const int i = (int)(t_ - r3_ * w3_), j = (int)(r3_ - q3_ * h3_), k = (int)q3_

template <class T>
__global__ void __launch_bounds__(256) m3_bcc_kernel(const M3Const<T> c, const Fields3<T> s, const Bcc3<T> b,
                                                     const int* __restrict__ active) {
    if (active && *active == 0) return;
    CC_FOR3(c.nx, c.ny, c.nz) {
        CC_IJK3(i, j, k);
        const size_t q = c.idx(i, j, k);
        b.x[q] = bx_cc3(c, s.bx, i, j, k);
        b.y[q] = by_cc3(c, s.by, i, j, k);
        b.z[q] = bz_cc3(c, s.bz, i, j, k);
    }
}

// ---------------------------------------------------------------------------
// primitives: 8 planes (rho, u, v, w, P, Bx, By, Bz)
template <class T> struct PrimData {
    T* w[8];
};

template <class T, bool DEFER>
__global__ void __launch_bounds__(256) m3_prim_kernel(const M3Const<T> c, const Fields3<T> s, const PrimData<T> pr,
                                                       const Bcc3<T> bcc, const double* __restrict__ dtp,
                                                       const int* __restrict__ active) {
    if (active && *active == 0) return;
    const T dt = (T)(*dtp);
    CC_FOR3(c.nx, c.ny, c.nz) {
        CC_IJK3(i, j, k);
        const size_t q = c.idx(i, j, k);
        T rho = s.rho[q], mx = s.mx[q], my = s.my[q], mz = s.mz[q], E = s.E[q];
        const T Bx = bx_cc3(c, s.bx, i, j, k), By = by_cc3(c, s.by, i, j, k), Bz = bz_cc3(c, s.bz, i, j, k);
        if (DEFER) {
            if (c.resistive) E += joule3_cc(c, bcc, i, j, k, dt);   // bcc: the cell-centred B of s
            floors(c, rho, mx, my, mz, E, Bx, By, Bz);  // M3:1019-1029
            s.rho[q] = rho;
            s.E[q] = E;
        }
        const Prim<T> W = to_prim(c, rho, mx, my, mz, E, Bx, By, Bz);
        pr.w[0][q] = W.r; pr.w[1][q] = W.u; pr.w[2][q] = W.v; pr.w[3][q] = W.w;
        pr.w[4][q] = W.P; pr.w[5][q] = W.bx; pr.w[6][q] = W.by; pr.w[7][q] = W.bz;
    }
}

// MUSCL-MC face state of cell q along (stride) with neighbours qm, qp:
// side +1 -> state at the cell's upper face, -1 -> lower face (M3:312-382).
// dir selects which B components are reconstructed (the normal one is not).
template <class T>
__device__ __forceinline__ Prim<T> face_state3(const PrimData<T>& pr, size_t qm, size_t q, size_t qp, int dir, T side,
                                               T floor_rho, T floor_P) {
    Prim<T> W;
    const T h = T(0.5) * side;
    auto rec = [&](int m) { return pr.w[m][q] + h * mc_slope(pr.w[m][qm], pr.w[m][q], pr.w[m][qp]); };
    W.r = rec(0); W.u = rec(1); W.v = rec(2); W.w = rec(3); W.P = rec(4);
    W.bx = (dir == 0) ? pr.w[5][q] : rec(5);
    W.by = (dir == 1) ? pr.w[6][q] : rec(6);
    W.bz = (dir == 2) ? pr.w[7][q] : rec(7);
    W.r = vmax(W.r, floor_rho);
    W.P = vmax(W.P, floor_P);
    return W;
}

// Faces of direction DIR (0 x, 1 y, 2 z): HLLD flux and face EMFs
// (M3:728-800).  Output slots: f[0..4] fluxes of rho, mx, my, mz, E;
// x: f[5] = Ey_x = F(Bz), f[6] = Ez_x = -F(By)
// y: f[5] = Ez_y = G(Bx), f[6] = Ex_y = -G(Bz)
// z: f[5] = Ex_z = H(By), f[6] = Ey_z = -H(Bx)
template <class T, int DIR>
__global__ void __launch_bounds__(256) m3_face_kernel(const M3Const<T> c, const Fields3<T> s, const PrimData<T> pr,
                                                      const FaceData<T> out, const int* __restrict__ active) {
    if (active && *active == 0) return;
    const int fx = c.nx + (DIR == 0), fy = c.ny + (DIR == 1), fz = c.nz + (DIR == 2);
    CC_FOR3(fx, fy, fz) {
        CC_IJK3(i, j, k);
        int Li = i, Lj = j, Lk = k, Ri = i, Rj = j, Rk = k;
        if (DIR == 0) { Li = c.ax.cell(i - 1); Ri = c.ax.cell(i); }
        if (DIR == 1) { Lj = c.ay.cell(j - 1); Rj = c.ay.cell(j); }
        if (DIR == 2) { Lk = c.az.cell(k - 1); Rk = c.az.cell(k); }
        // stencil neighbours of each side's cell, wrapped again from the wrapped index
        auto nb = [&](int a, int b, int d, int o) -> size_t {
            if (DIR == 0) return c.idx(c.ax.cell(a + o), b, d);
            if (DIR == 1) return c.idx(a, c.ay.cell(b + o), d);
            return c.idx(a, b, c.az.cell(d + o));
        };
        const Prim<T> WL = face_state3(pr, nb(Li, Lj, Lk, -1), c.idx(Li, Lj, Lk), nb(Li, Lj, Lk, +1), DIR, T(1),
                                       c.floor_rho, c.floor_P);
        const Prim<T> WR = face_state3(pr, nb(Ri, Rj, Rk, -1), c.idx(Ri, Rj, Rk), nb(Ri, Rj, Rk, +1), DIR, T(-1),
                                       c.floor_rho, c.floor_P);
        const size_t qf = c.idx(i, j, k);
        Flux<T> F;
        T e1, e2;
        if (DIR == 0) {
            F = hlld_x(c, WL, WR, s.bx[qf]);
            e1 = F.f6; e2 = -F.f5;
        } else if (DIR == 1) {
            F = hlld_y(c, WL, WR, s.by[qf]);
            e1 = F.f5; e2 = -F.f6;
        } else {
            F = hlld_z(c, WL, WR, s.bz[qf]);
            e1 = F.f6; e2 = -F.f5;
        }
        out.f[0][qf] = F.f0; out.f[1][qf] = F.f1; out.f[2][qf] = F.f2; out.f[3][qf] = F.f3; out.f[4][qf] = F.f4;
        out.f[5][qf] = e1; out.f[6][qf] = e2;
    }
}

// y (DIR 1) or z (DIR 2) faces as a march: a thread owns the (i, k) or (i, j)
// column and walks M3_FACE_MCH faces along the normal axis, holding the
// primitives of cells m-1, m, m+1 and the MC slopes of cells m-1 and m, so a
// cell's slopes are formed once for its two faces and each step loads one new
// cell.  Every face state is the same expression of the same values as in
// m3_face_kernel, where the stencil neighbours of a side's cell are re-mapped
// from its mapped index: on a periodic axis that equals the window; on a
// clamped one it differs only at the boundary faces (0 and n), which take the
// original path.
constexpr int M3_FACE_MCH = 32;
// (FP32 only) capped at 64 registers, four CTAs per SM: a few spilled values
// cost less than the latency a 98-register, two-CTA launch leaves exposed
// (256^3 FP32 step 7.26 -> 6.74 ms; 80 registers without spills: 6.80 ms)
template <class T, int DIR>
__global__ void __launch_bounds__(256, 4) m3_face_march_kernel(const M3Const<T> c, const Fields3<T> s,
                                                            const PrimData<T> pr, const FaceData<T> out,
                                                            const int* __restrict__ active) {
    static_assert(DIR == 1 || DIR == 2, "march along y or z");
    if (active && *active == 0) return;
    const int i = blockIdx.x * 32 + (threadIdx.x & 31), o = blockIdx.y * 8 + (threadIdx.x >> 5);
    const int n = DIR == 1 ? c.ny : c.nz, on = DIR == 1 ? c.nz : c.ny;
    if (i >= c.nx || o >= on) return;
    const AxisMap A = DIR == 1 ? c.ay : c.az;
    const int m0 = blockIdx.z * M3_FACE_MCH, m1 = min(n + 1, m0 + M3_FACE_MCH);
    auto cq = [&](int m) -> size_t { return DIR == 1 ? c.idx(i, A.cell(m), o) : c.idx(i, o, A.cell(m)); };
    const T hL = T(0.5) * T(1), hR = T(0.5) * T(-1);
    T w[3][8];    // cells m-1, m, m+1
    T sl[2][8];   // slopes of cells m-1, m (the normal B component has none)
    auto load = [&](T* d, int m) {
        const size_t q = cq(m);
#pragma unroll
        for (int k = 0; k < 8; k++) d[k] = pr.w[k][q];
    };
    auto slopes = [&](T* d, const T* a, const T* b, const T* e) {
#pragma unroll
        for (int k = 0; k < 8; k++) d[k] = mc_slope(a[k], b[k], e[k]);
    };
    T wm2[8];
    load(wm2, m0 - 2);
    load(w[0], m0 - 1);
    load(w[1], m0);
    load(w[2], m0 + 1);
    slopes(sl[0], wm2, w[0], w[1]);
    slopes(sl[1], w[0], w[1], w[2]);
    for (int m = m0; m < m1; ++m) {
        Prim<T> WL, WR;
        if (!A.periodic && (m == 0 || m == n)) {   // the boundary faces of a clamped axis: the original stencil
            const int Lc = A.cell(m - 1), Rc = A.cell(m);
            auto at = [&](int mm) -> size_t { return DIR == 1 ? c.idx(i, mm, o) : c.idx(i, o, mm); };
            WL = face_state3(pr, at(A.cell(Lc - 1)), at(Lc), at(A.cell(Lc + 1)), DIR, T(1), c.floor_rho, c.floor_P);
            WR = face_state3(pr, at(A.cell(Rc - 1)), at(Rc), at(A.cell(Rc + 1)), DIR, T(-1), c.floor_rho, c.floor_P);
        } else {
            auto side = [&](const T* v, const T* d, T h) {
                Prim<T> W;
                W.r = v[0] + h * d[0]; W.u = v[1] + h * d[1]; W.v = v[2] + h * d[2]; W.w = v[3] + h * d[3];
                W.P = v[4] + h * d[4];
                W.bx = v[5] + h * d[5];
                W.by = (DIR == 1) ? v[6] : v[6] + h * d[6];
                W.bz = (DIR == 2) ? v[7] : v[7] + h * d[7];
                W.r = vmax(W.r, c.floor_rho);
                W.P = vmax(W.P, c.floor_P);
                return W;
            };
            WL = side(w[0], sl[0], hL);
            WR = side(w[1], sl[1], hR);
        }
        const size_t qf = DIR == 1 ? c.idx(i, m, o) : c.idx(i, o, m);
        Flux<T> F;
        T e1, e2;
        if (DIR == 1) {
            F = hlld_y(c, WL, WR, s.by[qf]);
            e1 = F.f5; e2 = -F.f6;
        } else {
            F = hlld_z(c, WL, WR, s.bz[qf]);
            e1 = F.f6; e2 = -F.f5;
        }
        out.f[0][qf] = F.f0; out.f[1][qf] = F.f1; out.f[2][qf] = F.f2; out.f[3][qf] = F.f3; out.f[4][qf] = F.f4;
        out.f[5][qf] = e1; out.f[6][qf] = e2;
        if (m + 1 < m1) {   // advance the window to face m+1
#pragma unroll
            for (int k = 0; k < 8; k++) { w[0][k] = w[1][k]; w[1][k] = w[2][k]; sl[0][k] = sl[1][k]; }
            load(w[2], m + 2);
            slopes(sl[1], w[0], w[1], w[2]);
        }
    }
}

// FV update + floors with the stage-input B (M3:803-834)
template <class T>
__global__ void __launch_bounds__(256) m3_update_kernel(const M3Const<T> c, const Fields3<T> in, const Fields3<T> out,
                                                        const FaceData<T> X, const FaceData<T> Y, const FaceData<T> Z,
                                                        const double* __restrict__ dtp, const int* __restrict__ active) {
    if (active && *active == 0) return;
    const T dt = (T)(*dtp);
    CC_FOR3(c.nx, c.ny, c.nz) {
        CC_IJK3(i, j, k);
        const size_t q = c.idx(i, j, k), qx = c.idx(i + 1, j, k), qy = c.idx(i, j + 1, k), qz = c.idx(i, j, k + 1);
        T d[5];
#pragma unroll
        for (int m = 0; m < 5; m++)
            d[m] = -(X.f[m][qx] - X.f[m][q]) * c.inv_dx - (Y.f[m][qy] - Y.f[m][q]) * c.inv_dy -
                   (Z.f[m][qz] - Z.f[m][q]) * c.inv_dz;
        T rho = in.rho[q] + dt * d[0];
        T mx = in.mx[q] + dt * d[1];
        T my = in.my[q] + dt * d[2];
        T mz = in.mz[q] + dt * d[3];
        T E = in.E[q] + dt * d[4];
        floors(c, rho, mx, my, mz, E, bx_cc3(c, in.bx, i, j, k), by_cc3(c, in.by, i, j, k), bz_cc3(c, in.bz, i, j, k));
        out.rho[q] = rho; out.mx[q] = mx; out.my[q] = my; out.mz[q] = mz; out.E[q] = E;
    }
}

// Edge EMFs (M3:879-939): Balsara-Spicer average of the four face EMFs plus
// eta J from cell-centred B differences; Ex at (i, jf, kf), Ey at (if, j, kf),
// Ez at (if, jf, k).  EdgeColumn marches one (i, j) edge column in k,
// carrying what plane k-1 loaded (the EMF and cell-centred B at k-1, the
// z-face Bz at k); every value is the same expression of the same loads as a
// per-edge evaluation.
template <class T> struct EdgeColumn {
    const M3Const<T>& c;
    const Fields3<T>& in;
    const FaceData<T>& X;
    const FaceData<T>& Y;
    const FaceData<T>& Z;
    int i, j, ci, cim, fi, fi1, cj, cjm, fj, fj1;
    bool xe, ye, res_on;
    T exy_p, eyx_p, by_p, bx_p, bz0, bz0s, bz0w;

    __device__ __forceinline__ T at(const T* f, int a, int b, int d) const { return f[c.idx(a, b, d)]; }
    __device__ __forceinline__ T bxc(int jj, int kc) const { return T(0.5) * (at(in.bx, fi, jj, kc) + at(in.bx, fi1, jj, kc)); }
    __device__ __forceinline__ T byc(int ii, int kc) const { return T(0.5) * (at(in.by, ii, fj, kc) + at(in.by, ii, fj1, kc)); }

    // x-face EMF planes: X.f[5] = Ey_x, X.f[6] = Ez_x; y: Y.f[5] = Ez_y, Y.f[6] = Ex_y; z: Z.f[5] = Ex_z, Z.f[6] = Ey_z
    __device__ __forceinline__ EdgeColumn(const M3Const<T>& c_, const Fields3<T>& in_, const FaceData<T>& X_,
                                          const FaceData<T>& Y_, const FaceData<T>& Z_, int i_, int j_, int k0)
        : c(c_), in(in_), X(X_), Y(Y_), Z(Z_), i(i_), j(j_) {
        ci = c.ax.cell(i); cim = c.ax.cell(i - 1); fi = c.ax.face(i); fi1 = c.ax.face(i + 1);
        cj = c.ay.cell(j); cjm = c.ay.cell(j - 1); fj = c.ay.face(j); fj1 = c.ay.face(j + 1);
        xe = i < c.nx; ye = j < c.ny; res_on = c.resistive != 0;
        const int ckm = c.az.cell(k0 - 1), fk0 = c.az.face(k0);
        exy_p = at(Y.f[6], ci, fj, ckm); eyx_p = at(X.f[5], fi, cj, ckm);
        by_p = T(0); bx_p = T(0); bz0 = T(0); bz0s = T(0); bz0w = T(0);
        if (res_on) {
            by_p = byc(ci, ckm); bx_p = bxc(cj, ckm);
            bz0 = at(in.bz, ci, cj, fk0); bz0s = at(in.bz, ci, cjm, fk0); bz0w = at(in.bz, cim, cj, fk0);
        }
    }

    // the three EMFs of plane k (0 where the edge does not exist), then advance
    __device__ __forceinline__ void step(int k, T& ex, T& ey, T& ez) {
        const int ck = c.az.cell(k), fk = c.az.face(k), fk1 = c.az.face(k + 1);
        const T exy_k = at(Y.f[6], ci, fj, ck), eyx_k = at(X.f[5], fi, cj, ck);
        T by_k = T(0), bx_k = T(0), bz1 = T(0), bz1s = T(0), bz1w = T(0);
        if (res_on) {
            by_k = byc(ci, ck); bx_k = bxc(cj, ck);
            bz1 = at(in.bz, ci, cj, fk1); bz1s = at(in.bz, ci, cjm, fk1); bz1w = at(in.bz, cim, cj, fk1);
        }
        ex = ey = ez = T(0);
        if (xe) {  // Ex
            const T ideal = T(0.25) * (exy_p + exy_k + at(Z.f[5], ci, cjm, fk) + at(Z.f[5], ci, cj, fk));
            T res = T(0.0);
            if (res_on) {
                const T dBzdy = (T(0.5) * (bz0 + bz1) - T(0.5) * (bz0s + bz1s)) / c.dy;
                const T dBydz = (by_k - by_p) / c.dz;
                res = c.eta * (dBzdy - dBydz);
            }
            ex = ideal + res;
        }
        if (ye) {  // Ey
            const T ideal = T(0.25) * (eyx_p + eyx_k + at(Z.f[6], cim, cj, fk) + at(Z.f[6], ci, cj, fk));
            T res = T(0.0);
            if (res_on) {
                const T dBxdz = (bx_k - bx_p) / c.dz;
                const T dBzdx = (T(0.5) * (bz0 + bz1) - T(0.5) * (bz0w + bz1w)) / c.dx;
                res = c.eta * (dBxdz - dBzdx);
            }
            ey = ideal + res;
        }
        if (k < c.nz) {  // Ez
            const T ideal = T(0.25) * (at(X.f[6], fi, cjm, ck) + at(X.f[6], fi, cj, ck) + at(Y.f[5], cim, fj, ck) +
                                       at(Y.f[5], ci, fj, ck));
            T res = T(0.0);
            if (res_on) {
                const T dBydx = (by_k - byc(cim, ck)) / c.dx;
                const T dBxdy = (bx_k - bxc(cjm, ck)) / c.dy;
                res = c.eta * (dBydx - dBxdy);
            }
            ez = ideal + res;
        }
        exy_p = exy_k; eyx_p = eyx_k; by_p = by_k; bx_p = bx_k;
        bz0 = bz1; bz0s = bz1s; bz0w = bz1w;
    }
};

// Edge EMFs and the CT update of the three face arrays in one pass (M3:879-939
// then M3:942-1015).  A CTA of 32 x 8 threads owns the faces of 31 x 7 (i, j)
// columns over a chunk of M3_EDGE_KCH planes; each thread marches one edge
// column (EdgeColumn: the 32nd column and 8th row are the neighbours the
// owned faces read).  The march goes in bricks of M3_EMF_KB planes: a thread
// forms the EMFs of the brick's M3_EMF_KB + 1 edge planes (no barrier in
// between, so the loads of several planes are in flight together) into shared
// memory, then the owned faces of the brick's planes read their four edges
// there; the brick's last edge plane is the next brick's first.  So the edges
// never go to HBM (a stage no longer writes three edge planes and reads them
// back), and a brick costs two barriers.  The face update is the reference's
// expression of the same EMF values as before, so FP64 is unchanged bit for bit.
// Measured at 256^3 against the separate edge and CT kernels: FP32 step 6.67 ->
// 6.65 ms, FP64 16.32 -> 16.16 ms, three edge planes less memory (the edge
// march is latency-bound, and the saved traffic is small beside it); with a
// barrier pair per plane instead of per brick it was 1% slower.
constexpr int M3_EDGE_KCH = 32;
constexpr int M3_EMF_KB = 4;
template <class T>
__global__ void __launch_bounds__(256) m3_emf_ct_kernel(const M3Const<T> c, const Fields3<T> in, const Fields3<T> out,
                                                        const FaceData<T> X, const FaceData<T> Y, const FaceData<T> Z,
                                                        const double* __restrict__ dtp, const int* __restrict__ active) {
    if (active && *active == 0) return;
    constexpr int KB = M3_EMF_KB;
    __shared__ T sx[KB + 1][8][32], sy[KB + 1][8][32], sz[KB + 1][8][32];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int i = blockIdx.x * 31 + tx, j = blockIdx.y * 7 + ty;
    const bool live = i <= c.nx && j <= c.ny;
    const bool owner = live && tx < 31 && ty < 7;
    const int k0 = blockIdx.z * M3_EDGE_KCH;
    const int k1 = min(c.nz + 1, k0 + M3_EDGE_KCH);   // Bz planes k0 .. k1-1 of this chunk
    const int kend = min(k1, c.nz);                    // edge planes k0 .. kend
    const T dt = (T)(*dtp);
    const T dtdx = dt / c.dx, dtdy = dt / c.dy, dtdz = dt / c.dz;
    EdgeColumn<T> col(c, in, X, Y, Z, live ? i : 0, live ? j : 0, k0);
    for (int kb = k0; kb < k1; kb += KB) {
        // edge planes kb .. kb + KB into slots 0 .. KB (slot 0 carried from the last brick)
        if (kb > k0) {
            sx[0][ty][tx] = sx[KB][ty][tx]; sy[0][ty][tx] = sy[KB][ty][tx]; sz[0][ty][tx] = sz[KB][ty][tx];
        }
#pragma unroll
        for (int p = 0; p <= KB; ++p) {
            const int k = kb + p;
            if ((p > 0 || kb == k0) && k <= kend) {
                T ex = T(0), ey = T(0), ez = T(0);
                if (live) col.step(k, ex, ey, ez);
                sx[p][ty][tx] = ex; sy[p][ty][tx] = ey; sz[p][ty][tx] = ez;
            }
        }
        __syncthreads();
        if (owner) {
#pragma unroll
            for (int p = 0; p < KB; ++p) {
                const int kk = kb + p;
                if (kk >= k1) break;
                if (kk < kend) {   // Bx and By faces of plane kk (< nz): edge planes kk and kk + 1
                    const size_t q = c.idx(i, j, kk);
                    if (j < c.ny) {
                        const T ezU = sz[p][ty + 1][tx], ezD = sz[p][ty][tx];
                        const T eyF = sy[p + 1][ty][tx], eyB = sy[p][ty][tx];
                        out.bx[q] = in.bx[q] + (-(dtdy) * (ezU - ezD) + (dtdz) * (eyF - eyB));
                    }
                    if (i < c.nx) {
                        const T ezR = sz[p][ty][tx + 1], ezL = sz[p][ty][tx];
                        const T exF = sx[p + 1][ty][tx], exB = sx[p][ty][tx];
                        out.by[q] = in.by[q] + (+(dtdx) * (ezR - ezL) - (dtdz) * (exF - exB));
                    }
                }
                if (i < c.nx && j < c.ny) {   // Bz face of plane kk
                    const size_t q = c.idx(i, j, kk);
                    const T eyR = sy[p][ty][tx + 1], eyL = sy[p][ty][tx];
                    const T exU = sx[p][ty + 1][tx], exD = sx[p][ty][tx];
                    out.bz[q] = in.bz[q] + (-(dtdx) * (eyR - eyL) + (dtdy) * (exU - exD));
                }
            }
        }
        __syncthreads();   // slots are rewritten by the next brick
    }
}

// CFL speeds of a cell in three directions (compute_dt loop body, M3:633-636)
template <class T>
__device__ __forceinline__ double speed3(const M3Const<T>& c, const Prim<T>& W) {
    const T sx = fabs(W.u) + fast_speed(c, W, W.bx);
    const T sy = fabs(W.v) + fast_speed(c, W, W.by);
    const T sz = fabs(W.w) + fast_speed(c, W, W.bz);
    // std::max(maxs, x) ignores NaN x; keep each finite value
    double m = 0.0;
    if ((double)sx > m) m = (double)sx;
    if ((double)sy > m) m = (double)sy;
    if ((double)sz > m) m = (double)sz;
    return m;
}

// RK average (M3:1042-1065) with the deferred stage-2 Joule sub-step; emits the
// CFL and density partials of U^{n+1}.  Inactive: U^n carried over.
template <class T, int NT>
__global__ void __launch_bounds__(NT)
m3_average_kernel(const M3Const<T> c, const Fields3<T> un, const Fields3<T> s2, const Fields3<T> out,
                  const Bcc3<T> bcc, const double* __restrict__ dtp, const int* __restrict__ active,
                  double* __restrict__ spd_part, double* __restrict__ rho_part) {
    const bool act = (active == nullptr) || (*active != 0);
    __shared__ double sh[NT / 32];
    const T dt = (T)(*dtp);
    double smax = 0.0, rsum = 0.0;
    CC_FOR3(c.nx + 1, c.ny + 1, c.nz + 1) {
        CC_IJK3(i, j, k);
        const size_t q = c.idx(i, j, k);
        auto avx = [&](size_t f) { return act ? T(0.5) * (un.bx[f] + s2.bx[f]) : un.bx[f]; };
        auto avy = [&](size_t f) { return act ? T(0.5) * (un.by[f] + s2.by[f]) : un.by[f]; };
        auto avz = [&](size_t f) { return act ? T(0.5) * (un.bz[f] + s2.bz[f]) : un.bz[f]; };
        if (j < c.ny && k < c.nz) out.bx[q] = avx(q);
        if (i < c.nx && k < c.nz) out.by[q] = avy(q);
        if (i < c.nx && j < c.ny) out.bz[q] = avz(q);
        if (i >= c.nx || j >= c.ny || k >= c.nz) continue;
        const T Bx = T(0.5) * (avx(q) + avx(c.idx(i + 1, j, k)));
        const T By = T(0.5) * (avy(q) + avy(c.idx(i, j + 1, k)));
        const T Bz = T(0.5) * (avz(q) + avz(c.idx(i, j, k + 1)));
        T rho, mx, my, mz, E;
        if (act) {
            T r2 = s2.rho[q], m2x = s2.mx[q], m2y = s2.my[q], m2z = s2.mz[q], E2 = s2.E[q];
            if (c.resistive) E2 += joule3_cc(c, bcc, i, j, k, dt);   // bcc: the cell-centred B of s2
            floors(c, r2, m2x, m2y, m2z, E2, bx_cc3(c, s2.bx, i, j, k), by_cc3(c, s2.by, i, j, k),
                   bz_cc3(c, s2.bz, i, j, k));
            rho = T(0.5) * (un.rho[q] + r2);
            mx = T(0.5) * (un.mx[q] + m2x);
            my = T(0.5) * (un.my[q] + m2y);
            mz = T(0.5) * (un.mz[q] + m2z);
            E = T(0.5) * (un.E[q] + E2);
            floors(c, rho, mx, my, mz, E, Bx, By, Bz);
        } else {
            rho = un.rho[q]; mx = un.mx[q]; my = un.my[q]; mz = un.mz[q]; E = un.E[q];
        }
        out.rho[q] = rho; out.mx[q] = mx; out.my[q] = my; out.mz[q] = mz; out.E[q] = E;
        const Prim<T> W = to_prim(c, rho, mx, my, mz, E, Bx, By, Bz);
        const double s = speed3(c, W);
        if (s > smax) smax = s;
        rsum += (double)rho;
    }
    const double bm = block_max<NT>(smax, sh);
    const double bs = block_sum<NT>(rsum, sh);
    if (threadIdx.x == 0) { spd_part[blockIdx.x] = bm; rho_part[blockIdx.x] = bs; }
}

template <class T, int NT>
__global__ void __launch_bounds__(NT)
m3_speed_kernel(const M3Const<T> c, const Fields3<T> s, double* __restrict__ spd_part) {
    __shared__ double sh[NT / 32];
    double smax = 0.0;
    CC_FOR3(c.nx, c.ny, c.nz) {
        CC_IJK3(i, j, k);
        const size_t q = c.idx(i, j, k);
        const Prim<T> W = to_prim(c, s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc3(c, s.bx, i, j, k),
                                  by_cc3(c, s.by, i, j, k), bz_cc3(c, s.bz, i, j, k));
        const double v = speed3(c, W);
        if (v > smax) smax = v;
    }
    const double bm = block_max<NT>(smax, sh);
    if (threadIdx.x == 0) spd_part[blockIdx.x] = bm;
}

// FP64 sums (rho, mx, my, mz, E), max |div B| (M3:1070-1078), non-finite flag
template <class T, int NT>
__global__ void __launch_bounds__(NT) m3_diag_kernel(const M3Const<T> c, const Fields3<T> s, double* __restrict__ part) {
    __shared__ double sh[NT / 32];
    double acc[5] = {0, 0, 0, 0, 0}, dmax = 0.0, nonf = 0.0;
    CC_FOR3(c.nx, c.ny, c.nz) {
        CC_IJK3(i, j, k);
        const size_t q = c.idx(i, j, k);
        const double v[5] = {(double)s.rho[q], (double)s.mx[q], (double)s.my[q], (double)s.mz[q], (double)s.E[q]};
        for (int m = 0; m < 5; m++) {
            acc[m] += v[m];
            if (!isfinite(v[m])) nonf = 1.0;
        }
        const double d = ((double)s.bx[c.idx(i + 1, j, k)] - (double)s.bx[q]) / (double)c.dx +
                         ((double)s.by[c.idx(i, j + 1, k)] - (double)s.by[q]) / (double)c.dy +
                         ((double)s.bz[c.idx(i, j, k + 1)] - (double)s.bz[q]) / (double)c.dz;
        dmax = fmax(dmax, fabs(d));
    }
    for (int m = 0; m < 5; m++) {
        const double b = block_sum<NT>(acc[m], sh);
        if (threadIdx.x == 0) part[m * gridDim.x + blockIdx.x] = b;
    }
    const double bm = block_max<NT>(dmax, sh);
    const double bn = block_max<NT>(nonf, sh);
    if (threadIdx.x == 0) { part[5 * gridDim.x + blockIdx.x] = bm; part[6 * gridDim.x + blockIdx.x] = bn; }
}

// Snapshot fields of the reference main()'s store (M3:1293-1321), in its
// order: rho, P, Mach, u, v, w, vabs, Bx, By, Bz (cell-centred, from the
// faces), div B; out: 11 planes of nx*ny*nz doubles, x fastest.
// cs = sqrt(sound_speed2) (hybrid EOS), Mach = |v| / max(cs, 1e-12); div B in FP64.
template <class T>
__global__ void m3_derived_kernel(const M3Const<T> c, const Fields3<T> s, double* __restrict__ out) {
    const size_t n = (size_t)c.nx * c.ny * c.nz;
    CC_FOR3(c.nx, c.ny, c.nz) {
        CC_IJK3(i, j, k);
        const size_t q = c.idx(i, j, k), o = (size_t)t_;
        const T Bx = T(0.5) * (s.bx[q] + s.bx[c.idx(i + 1, j, k)]);
        const T By = T(0.5) * (s.by[q] + s.by[c.idx(i, j + 1, k)]);
        const T Bz = T(0.5) * (s.bz[q] + s.bz[c.idx(i, j, k + 1)]);
        const Prim<T> W = to_prim(c, s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], Bx, By, Bz);
        const T cs = sqrt(sound_speed2(c, W));
        const T vabs = sqrt(W.u * W.u + W.v * W.v + W.w * W.w);
        const T mach = vabs / vmax(cs, T(1e-12));
        const double div = ((double)s.bx[c.idx(i + 1, j, k)] - (double)s.bx[q]) / (double)c.dx +
                           ((double)s.by[c.idx(i, j + 1, k)] - (double)s.by[q]) / (double)c.dy +
                           ((double)s.bz[c.idx(i, j, k + 1)] - (double)s.bz[q]) / (double)c.dz;
        const double v[11] = {(double)W.r, (double)W.P, (double)mach, (double)W.u, (double)W.v, (double)W.w,
                              (double)vabs, (double)W.bx, (double)W.by, (double)W.bz, div};
#pragma unroll
        for (int m = 0; m < 11; m++) out[m * n + o] = v[m];
    }
}

// host layout (x fastest, w x h x d) <-> pitched 3D field
template <class T>
__global__ void pack3_in_kernel(const double* __restrict__ src, T* __restrict__ dst, int w, int h, int d, int P,
                                long long PS) {
    CC_FOR3(w, h, d) {
        CC_IJK3(i, j, k);
        dst[(size_t)k * PS + (size_t)j * P + i] = (T)src[t_];
    }
}
template <class T>
__global__ void pack3_out_kernel(const T* __restrict__ src, double* __restrict__ dst, int w, int h, int d, int P,
                                 long long PS) {
    CC_FOR3(w, h, d) {
        CC_IJK3(i, j, k);
        dst[t_] = (double)src[(size_t)k * PS + (size_t)j * P + i];
    }
}

}  // namespace ccb
