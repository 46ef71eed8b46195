// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// CPU restatement of the 3D resistive-MHD step of mhd3d_resistive_hlld_ct.cpp
// (cited as M3:<line>): hybrid cold + thermal EOS with bounce stiffening,
// MUSCL-MC, HLLD in x/y/z, arithmetic-average edge EMFs with eta J from
// cell-centred B, CT, Joule heating, SSP-RK2.  One loop per reference sub-step.
#pragma once
#include <array>
#include <cmath>
#include <vector>

#include "oracle_common.hpp"

namespace cco {

struct M3Par {
    double gamma1, gamma2, K1, rho_nuc, gamma_th, rho_bounce, gamma_bounce, Kbounce;
    double cfl, x0, x1, y0, y1, z0, z1;
    int nx, ny, nz;
    double floor_rho, floor_P;
    bool px, py, pz;
    double eta;
    double dx() const { return (x1 - x0) / nx; }
    double dy() const { return (y1 - y0) / ny; }
    double dz() const { return (z1 - z0) / nz; }
};

template <class T> struct M3State {
    std::vector<T> rho, mx, my, mz, E;  // (k*ny + j)*nx + i
    std::vector<T> bxf;                 // (k*ny + j)*(nx+1) + i_face
    std::vector<T> byf;                 // (k*(ny+1) + j_face)*nx + i
    std::vector<T> bzf;                 // (k_face*ny + j)*nx + i
};

template <class T> struct Cold { T P, e, g; };

template <class T> class M3 {
public:
    M3Par p;
    Axis ax, ay, az;
    explicit M3(const M3Par& par) : p(par), ax{par.nx, par.px}, ay{par.ny, par.py}, az{par.nz, par.pz} {}

    // ---- hybrid EOS (M3:116-212) ----
    Cold<T> cold(T rho) const {
        rho = vmax(rho, T(p.floor_rho));
        const T g1 = T(p.gamma1), g2 = T(p.gamma2), K1 = T(p.K1), rn = T(p.rho_nuc);
        T K2 = K1 * std::pow(rn, g1 - g2);
        if (rho < rn) {
            T Pc = K1 * std::pow(rho, g1);
            T ec = K1 * std::pow(rho, g1 - T(1.0)) / (g1 - T(1.0));
            return {Pc, ec, g1};
        }
        T Pc = K2 * std::pow(rho, g2);
        T e1 = K1 * std::pow(rn, g1 - T(1.0)) / (g1 - T(1.0));
        T e2 = K2 * std::pow(rn, g2 - T(1.0)) / (g2 - T(1.0));
        T ec = e1 + (K2 * std::pow(rho, g2 - T(1.0)) / (g2 - T(1.0)) - e2);
        T gc = g2;
        const T rb = T(p.rho_bounce), gb = T(p.gamma_bounce), Kb = T(p.Kbounce);
        if (rho >= rb) {
            T pb = Kb * (std::pow(rho, gb) - std::pow(rb, gb));
            T eb = Kb * (std::pow(rho, gb - T(1.0)) - std::pow(rb, gb - T(1.0))) / (gb - T(1.0));
            Pc += pb;
            ec += eb;
            gc = (g2 * (Pc - pb) + gb * pb) / vmax(Pc, T(p.floor_P));
        }
        return {Pc, ec, gc};
    }
    T pressure(T rho, T e_spec) const {
        rho = vmax(rho, T(p.floor_rho));
        Cold<T> c = cold(rho);
        T eth = vmax(T(0.0), e_spec - c.e);
        T Pth = (T(p.gamma_th) - T(1.0)) * rho * eth;
        return vmax(c.P + Pth, T(p.floor_P));
    }
    T energy(const Prim8<T>& W) const {  // total_energy_from_prim (M3:154-163)
        T rho = vmax(W.r, T(p.floor_rho));
        T kin = T(0.5) * rho * (W.u * W.u + W.v * W.v + W.w * W.w);
        T mag = T(0.5) * (W.bx * W.bx + W.by * W.by + W.bz * W.bz);
        Cold<T> c = cold(rho);
        T Pth = vmax(T(0.0), W.P - c.P);
        T eth = (T(p.gamma_th) > T(1.0)) ? (Pth / ((T(p.gamma_th) - T(1.0)) * rho)) : T(0.0);
        T eint = rho * (c.e + eth);
        return kin + mag + eint;
    }
    void floors(T& rho, T& mx, T& my, T& mz, T& E, T Bx, T By, T Bz) const {  // M3:165-183
        rho = vmax(rho, T(p.floor_rho));
        T u = mx / rho, v = my / rho, w = mz / rho;
        T kin = T(0.5) * rho * (u * u + v * v + w * w);
        T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
        T eint = E - kin - mag;
        if (eint < T(0.0)) eint = T(0.0);
        T es = eint / rho;
        T P = pressure(rho, es);
        if (P < T(p.floor_P)) P = T(p.floor_P);
        Cold<T> c = cold(rho);
        T Pth = vmax(T(0.0), P - c.P);
        T eth = (T(p.gamma_th) > T(1.0)) ? (Pth / ((T(p.gamma_th) - T(1.0)) * rho)) : T(0.0);
        T en = rho * (c.e + eth);
        E = kin + mag + en;
    }
    Prim8<T> to_prim(T rho, T mx, T my, T mz, T E, T Bx, T By, T Bz) const {  // M3:185-197
        rho = vmax(rho, T(p.floor_rho));
        T u = mx / rho, v = my / rho, w = mz / rho;
        T kin = T(0.5) * rho * (u * u + v * v + w * w);
        T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
        T eint = E - kin - mag;
        if (eint < T(0.0)) eint = T(0.0);
        T es = eint / rho;
        T P = pressure(rho, es);
        if (P < T(p.floor_P)) P = T(p.floor_P);
        return {rho, u, v, w, P, Bx, By, Bz};
    }
    T a2(const Prim8<T>& W) const {  // sound_speed2 (M3:206-212)
        T rho = vmax(W.r, T(p.floor_rho));
        Cold<T> c = cold(rho);
        T Pth = vmax(T(0.0), W.P - c.P);
        T num = c.g * c.P + T(p.gamma_th) * Pth;
        return vmax(T(0.0), num / rho);
    }
    T fast(const Prim8<T>& W, T bn2) const {  // fast_speed_x/y/z (M3:214-248)
        T s2 = a2(W);
        T b2 = W.bx * W.bx + W.by * W.by + W.bz * W.bz;
        T rho = vmax(W.r, T(1e-300));
        T vA2 = b2 / rho;
        T vn2 = bn2 / rho;
        T disc = (s2 + vA2) * (s2 + vA2) - T(4.0) * s2 * vn2;
        disc = vmax(T(0.0), disc);
        T cf2 = T(0.5) * ((s2 + vA2) + std::sqrt(disc));
        return std::sqrt(vmax(T(0.0), cf2));
    }

    // ---- indexing with the reference's wrap rules (M3:250-308) ----
    size_t cid(int i, int j, int k) const { return ((size_t)k * p.ny + j) * p.nx + i; }
    T bxf(const M3State<T>& s, int i, int j, int k) const {
        return s.bxf[((size_t)az.cell(k) * p.ny + ay.cell(j)) * (p.nx + 1) + ax.face(i)];
    }
    T byf(const M3State<T>& s, int i, int j, int k) const {
        return s.byf[((size_t)az.cell(k) * (p.ny + 1) + ay.face(j)) * p.nx + ax.cell(i)];
    }
    T bzf(const M3State<T>& s, int i, int j, int k) const {
        return s.bzf[((size_t)az.face(k) * p.ny + ay.cell(j)) * p.nx + ax.cell(i)];
    }
    // cell-centred B from unwrapped indices: the face lookups wrap, so at a
    // periodic seam the normal component averages faces N and 0 (M3:280-296)
    T bx_cc(const M3State<T>& s, int i, int j, int k) const { return T(0.5) * (bxf(s, i, j, k) + bxf(s, i + 1, j, k)); }
    T by_cc(const M3State<T>& s, int i, int j, int k) const { return T(0.5) * (byf(s, i, j, k) + byf(s, i, j + 1, k)); }
    T bz_cc(const M3State<T>& s, int i, int j, int k) const { return T(0.5) * (bzf(s, i, j, k) + bzf(s, i, j, k + 1)); }
    Prim8<T> prim_at(const M3State<T>& s, int i, int j, int k) const {  // get_prim_cc (M3:298-308)
        i = ax.cell(i); j = ay.cell(j); k = az.cell(k);
        size_t q = cid(i, j, k);
        return to_prim(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc(s, i, j, k), by_cc(s, i, j, k),
                       bz_cc(s, i, j, k));
    }

    // MUSCL-MC along dir (0 x, 1 y, 2 z) of the (already wrapped) cell (M3:312-382)
    void recon(const M3State<T>& s, int i, int j, int k, int dir, Prim8<T>& WL, Prim8<T>& WR) const {
        int di = dir == 0, dj = dir == 1, dk = dir == 2;
        Prim8<T> Wm = prim_at(s, i - di, j - dj, k - dk), Wc = prim_at(s, i, j, k), Wp = prim_at(s, i + di, j + dj, k + dk);
        auto lim = [&](T wm, T wc, T wp) { return mc_slope(wc - wm, wp - wc); };
        T sr = lim(Wm.r, Wc.r, Wp.r), su = lim(Wm.u, Wc.u, Wp.u), sv = lim(Wm.v, Wc.v, Wp.v);
        T sw = lim(Wm.w, Wc.w, Wp.w), sP = lim(Wm.P, Wc.P, Wp.P);
        WL = Wc; WR = Wc;
        WL.r = Wc.r - T(0.5) * sr; WR.r = Wc.r + T(0.5) * sr;
        WL.u = Wc.u - T(0.5) * su; WR.u = Wc.u + T(0.5) * su;
        WL.v = Wc.v - T(0.5) * sv; WR.v = Wc.v + T(0.5) * sv;
        WL.w = Wc.w - T(0.5) * sw; WR.w = Wc.w + T(0.5) * sw;
        WL.P = Wc.P - T(0.5) * sP; WR.P = Wc.P + T(0.5) * sP;
        if (dir != 0) { T sb = lim(Wm.bx, Wc.bx, Wp.bx); WL.bx = Wc.bx - T(0.5) * sb; WR.bx = Wc.bx + T(0.5) * sb; }
        if (dir != 1) { T sb = lim(Wm.by, Wc.by, Wp.by); WL.by = Wc.by - T(0.5) * sb; WR.by = Wc.by + T(0.5) * sb; }
        if (dir != 2) { T sb = lim(Wm.bz, Wc.bz, Wp.bz); WL.bz = Wc.bz - T(0.5) * sb; WR.bz = Wc.bz + T(0.5) * sb; }
        WL.r = vmax(WL.r, T(p.floor_rho)); WR.r = vmax(WR.r, T(p.floor_rho));
        WL.P = vmax(WL.P, T(p.floor_P));   WR.P = vmax(WR.P, T(p.floor_P));
    }

    Flux7<T> hlld_x(Prim8<T> L, Prim8<T> R, T Bn) const { return hlld_x_generic(*this, L, R, Bn); }
    // y: swap (u,v),(Bx,By) (M3:577-595); out f1 = F(mx), f2 = F(my), f5 = F(Bx), f6 = F(Bz)
    Flux7<T> hlld_y(Prim8<T> L, Prim8<T> R, T Bn) const {
        L.by = Bn; R.by = Bn;
        Prim8<T> aL{L.r, L.v, L.u, L.w, L.P, L.by, L.bx, L.bz};
        Prim8<T> aR{R.r, R.v, R.u, R.w, R.P, R.by, R.bx, R.bz};
        Flux7<T> F = hlld_x(aL, aR, Bn), G = F;
        G.f[1] = F.f[2]; G.f[2] = F.f[1];
        return G;
    }
    // z: cyclic (w,u,v),(Bz,Bx,By) (M3:604-622); out f1 = F(mx), f2 = F(my), f3 = F(mz), f5 = F(Bx), f6 = F(By)
    Flux7<T> hlld_z(Prim8<T> L, Prim8<T> R, T Bn) const {
        L.bz = Bn; R.bz = Bn;
        Prim8<T> aL{L.r, L.w, L.u, L.v, L.P, L.bz, L.bx, L.by};
        Prim8<T> aR{R.r, R.w, R.u, R.v, R.P, R.bz, R.bx, R.by};
        Flux7<T> F = hlld_x(aL, aR, Bn), H = F;
        H.f[1] = F.f[2]; H.f[2] = F.f[3]; H.f[3] = F.f[1];
        return H;
    }

    // advance_stage (M3:694-1030)
    void advance_stage(const M3State<T>& s0, M3State<T>& s1, T dt) const {
        const int nx = p.nx, ny = p.ny, nz = p.nz;
        const T dx = T(p.dx()), dy = T(p.dy()), dz = T(p.dz());
        s1 = s0;
        auto fx = [&](int i, int j, int k) { return ((size_t)k * ny + j) * (nx + 1) + i; };
        auto fy = [&](int i, int j, int k) { return ((size_t)k * (ny + 1) + j) * nx + i; };
        auto fz = [&](int i, int j, int k) { return ((size_t)k * ny + j) * nx + i; };
        std::vector<Flux7<T>> Fx((size_t)(nx + 1) * ny * nz), Gy((size_t)nx * (ny + 1) * nz), Hz((size_t)nx * ny * (nz + 1));
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i <= nx; i++) {
                    Prim8<T> a, WL, WR, b;
                    recon(s0, ax.cell(i - 1), j, k, 0, a, WL);
                    recon(s0, ax.cell(i), j, k, 0, WR, b);
                    Fx[fx(i, j, k)] = hlld_x(WL, WR, bxf(s0, i, j, k));
                }
        for (int k = 0; k < nz; k++)
            for (int j = 0; j <= ny; j++)
                for (int i = 0; i < nx; i++) {
                    Prim8<T> a, WL, WR, b;
                    recon(s0, i, ay.cell(j - 1), k, 1, a, WL);
                    recon(s0, i, ay.cell(j), k, 1, WR, b);
                    Gy[fy(i, j, k)] = hlld_y(WL, WR, byf(s0, i, j, k));
                }
        for (int k = 0; k <= nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    Prim8<T> a, WL, WR, b;
                    recon(s0, i, j, az.cell(k - 1), 2, a, WL);
                    recon(s0, i, j, az.cell(k), 2, WR, b);
                    Hz[fz(i, j, k)] = hlld_z(WL, WR, bzf(s0, i, j, k));
                }
        // FV update + floors with the stage-input B (M3:803-834)
        const T idx = T(1.0) / dx, idy = T(1.0) / dy, idz = T(1.0) / dz;
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    size_t q = cid(i, j, k);
                    const Flux7<T>&R = Fx[fx(i + 1, j, k)], &L = Fx[fx(i, j, k)];
                    const Flux7<T>&U = Gy[fy(i, j + 1, k)], &D = Gy[fy(i, j, k)];
                    const Flux7<T>&F = Hz[fz(i, j, k + 1)], &B = Hz[fz(i, j, k)];
                    T d[5];
                    for (int m = 0; m < 5; m++)
                        d[m] = -(R.f[m] - L.f[m]) * idx - (U.f[m] - D.f[m]) * idy - (F.f[m] - B.f[m]) * idz;
                    s1.rho[q] += dt * d[0];
                    s1.mx[q] += dt * d[1];
                    s1.my[q] += dt * d[2];
                    s1.mz[q] += dt * d[3];
                    s1.E[q] += dt * d[4];
                    floors(s1.rho[q], s1.mx[q], s1.my[q], s1.mz[q], s1.E[q], bx_cc(s0, i, j, k), by_cc(s0, i, j, k),
                           bz_cc(s0, i, j, k));
                }
        // face EMFs: Ey_x = F(Bz), Ez_x = -F(By); Ez_y = G(Bx), Ex_y = -G(Bz);
        // Ex_z = H(By), Ey_z = -H(Bx)   (M3:746-747, 771-772, 796-797)
        auto exy = [&](int i, int j, int k) { return -Gy[fy(ax.cell(i), ay.face(j), az.cell(k))].f[6]; };
        auto ezx = [&](int i, int j, int k) { return -Fx[fx(ax.face(i), ay.cell(j), az.cell(k))].f[5]; };
        auto eyx = [&](int i, int j, int k) { return Fx[fx(ax.face(i), ay.cell(j), az.cell(k))].f[6]; };
        auto exz = [&](int i, int j, int k) { return Hz[fz(ax.cell(i), ay.cell(j), az.face(k))].f[6]; };
        auto eyz = [&](int i, int j, int k) { return -Hz[fz(ax.cell(i), ay.cell(j), az.face(k))].f[5]; };
        auto ezy = [&](int i, int j, int k) { return Gy[fy(ax.cell(i), ay.face(j), az.cell(k))].f[5]; };
        const T eta = T(p.eta);
        std::vector<T> Ex((size_t)nx * (ny + 1) * (nz + 1)), Ey((size_t)(nx + 1) * ny * (nz + 1)), Ez((size_t)(nx + 1) * (ny + 1) * nz);
        for (int kf = 0; kf <= nz; kf++)  // M3:879-897
            for (int jf = 0; jf <= ny; jf++)
                for (int i = 0; i < nx; i++) {
                    T ideal = T(0.25) * (exy(i, jf, kf - 1) + exy(i, jf, kf) + exz(i, jf - 1, kf) + exz(i, jf, kf));
                    T res = T(0.0);
                    if (p.eta > 0.0) {
                        T dBzdy = (bz_cc(s0, i, jf, kf) - bz_cc(s0, i, jf - 1, kf)) / dy;
                        T dBydz = (by_cc(s0, i, jf, kf) - by_cc(s0, i, jf, kf - 1)) / dz;
                        res = eta * (dBzdy - dBydz);
                    }
                    Ex[((size_t)kf * (ny + 1) + jf) * nx + i] = ideal + res;
                }
        for (int kf = 0; kf <= nz; kf++)  // M3:900-918
            for (int j = 0; j < ny; j++)
                for (int i = 0; i <= nx; i++) {
                    T ideal = T(0.25) * (eyx(i, j, kf - 1) + eyx(i, j, kf) + eyz(i - 1, j, kf) + eyz(i, j, kf));
                    T res = T(0.0);
                    if (p.eta > 0.0) {
                        T dBxdz = (bx_cc(s0, i, j, kf) - bx_cc(s0, i, j, kf - 1)) / dz;
                        T dBzdx = (bz_cc(s0, i, j, kf) - bz_cc(s0, i - 1, j, kf)) / dx;
                        res = eta * (dBxdz - dBzdx);
                    }
                    Ey[((size_t)kf * ny + j) * (nx + 1) + i] = ideal + res;
                }
        for (int k = 0; k < nz; k++)  // M3:921-939
            for (int jf = 0; jf <= ny; jf++)
                for (int i = 0; i <= nx; i++) {
                    T ideal = T(0.25) * (ezx(i, jf - 1, k) + ezx(i, jf, k) + ezy(i - 1, jf, k) + ezy(i, jf, k));
                    T res = T(0.0);
                    if (p.eta > 0.0) {
                        T dBydx = (by_cc(s0, i, jf, k) - by_cc(s0, i - 1, jf, k)) / dx;
                        T dBxdy = (bx_cc(s0, i, jf, k) - bx_cc(s0, i, jf - 1, k)) / dy;
                        res = eta * (dBydx - dBxdy);
                    }
                    Ez[((size_t)k * (ny + 1) + jf) * (nx + 1) + i] = ideal + res;
                }
        // CT (M3:942-1015)
        for (int k = 0; k < nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i <= nx; i++) {
                    int j0 = ay.face(j), j1 = ay.face(j + 1), k0 = az.face(k), k1 = az.face(k + 1);
                    T ezU = Ez[((size_t)k * (ny + 1) + j1) * (nx + 1) + i], ezD = Ez[((size_t)k * (ny + 1) + j0) * (nx + 1) + i];
                    T eyF = Ey[((size_t)k1 * ny + j) * (nx + 1) + i], eyB = Ey[((size_t)k0 * ny + j) * (nx + 1) + i];
                    s1.bxf[fx(i, j, k)] += -(dt / dy) * (ezU - ezD) + (dt / dz) * (eyF - eyB);
                }
        for (int k = 0; k < nz; k++)
            for (int j = 0; j <= ny; j++)
                for (int i = 0; i < nx; i++) {
                    int i0 = ax.face(i), i1 = ax.face(i + 1), k0 = az.face(k), k1 = az.face(k + 1);
                    T ezR = Ez[((size_t)k * (ny + 1) + j) * (nx + 1) + i1], ezL = Ez[((size_t)k * (ny + 1) + j) * (nx + 1) + i0];
                    T exF = Ex[((size_t)k1 * (ny + 1) + j) * nx + i], exB = Ex[((size_t)k0 * (ny + 1) + j) * nx + i];
                    s1.byf[fy(i, j, k)] += +(dt / dx) * (ezR - ezL) - (dt / dz) * (exF - exB);
                }
        for (int k = 0; k <= nz; k++)
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    int i0 = ax.face(i), i1 = ax.face(i + 1), j0 = ay.face(j), j1 = ay.face(j + 1);
                    T eyR = Ey[((size_t)k * ny + j) * (nx + 1) + i1], eyL = Ey[((size_t)k * ny + j) * (nx + 1) + i0];
                    T exU = Ex[((size_t)k * (ny + 1) + j1) * nx + i], exD = Ex[((size_t)k * (ny + 1) + j0) * nx + i];
                    s1.bzf[fz(i, j, k)] += -(dt / dx) * (eyR - eyL) + (dt / dy) * (exU - exD);
                }
        joule(s1, dt);
        for (int k = 0; k < nz; k++)  // M3:1019-1029
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    size_t q = cid(i, j, k);
                    floors(s1.rho[q], s1.mx[q], s1.my[q], s1.mz[q], s1.E[q], bx_cc(s1, i, j, k), by_cc(s1, i, j, k),
                           bz_cc(s1, i, j, k));
                }
    }

    // add_joule_heating (M3:652-692): J from central differences of
    // cell-centred B at unwrapped neighbour indices
    void joule(M3State<T>& s, T dt) const {
        if (!(p.eta > 0.0)) return;
        const T dx = T(p.dx()), dy = T(p.dy()), dz = T(p.dz()), eta = T(p.eta);
        for (int k = 0; k < p.nz; k++)
            for (int j = 0; j < p.ny; j++)
                for (int i = 0; i < p.nx; i++) {
                    T dBzdy = (bz_cc(s, i, j + 1, k) - bz_cc(s, i, j - 1, k)) / (T(2) * dy);
                    T dBydz = (by_cc(s, i, j, k + 1) - by_cc(s, i, j, k - 1)) / (T(2) * dz);
                    T dBxdz = (bx_cc(s, i, j, k + 1) - bx_cc(s, i, j, k - 1)) / (T(2) * dz);
                    T dBzdx = (bz_cc(s, i + 1, j, k) - bz_cc(s, i - 1, j, k)) / (T(2) * dx);
                    T dBydx = (by_cc(s, i + 1, j, k) - by_cc(s, i - 1, j, k)) / (T(2) * dx);
                    T dBxdy = (bx_cc(s, i, j + 1, k) - bx_cc(s, i, j - 1, k)) / (T(2) * dy);
                    T Jx = dBzdy - dBydz, Jy = dBxdz - dBzdx, Jz = dBydx - dBxdy;
                    T J2 = Jx * Jx + Jy * Jy + Jz * Jz;
                    s.E[cid(i, j, k)] += dt * eta * J2;
                }
    }

    void rk2_step(M3State<T>& s, T dt) const {  // M3:1034-1066
        M3State<T> s1, s2;
        advance_stage(s, s1, dt);
        advance_stage(s1, s2, dt);
        for (size_t q = 0; q < s.rho.size(); q++) {
            s.rho[q] = T(0.5) * (s.rho[q] + s2.rho[q]);
            s.mx[q] = T(0.5) * (s.mx[q] + s2.mx[q]);
            s.my[q] = T(0.5) * (s.my[q] + s2.my[q]);
            s.mz[q] = T(0.5) * (s.mz[q] + s2.mz[q]);
            s.E[q] = T(0.5) * (s.E[q] + s2.E[q]);
        }
        for (size_t q = 0; q < s.bxf.size(); q++) s.bxf[q] = T(0.5) * (s.bxf[q] + s2.bxf[q]);
        for (size_t q = 0; q < s.byf.size(); q++) s.byf[q] = T(0.5) * (s.byf[q] + s2.byf[q]);
        for (size_t q = 0; q < s.bzf.size(); q++) s.bzf[q] = T(0.5) * (s.bzf[q] + s2.bzf[q]);
        for (int k = 0; k < p.nz; k++)
            for (int j = 0; j < p.ny; j++)
                for (int i = 0; i < p.nx; i++) {
                    size_t q = cid(i, j, k);
                    floors(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc(s, i, j, k), by_cc(s, i, j, k), bz_cc(s, i, j, k));
                }
    }

    double compute_dt(const M3State<T>& s) const {  // M3:626-648
        double maxs = 1e-14;
        for (int k = 0; k < p.nz; k++)
            for (int j = 0; j < p.ny; j++)
                for (int i = 0; i < p.nx; i++) {
                    Prim8<T> W = prim_at(s, i, j, k);
                    maxs = vmax(maxs, (double)(std::abs(W.u) + fast(W, W.bx * W.bx)));
                    maxs = vmax(maxs, (double)(std::abs(W.v) + fast(W, W.by * W.by)));
                    maxs = vmax(maxs, (double)(std::abs(W.w) + fast(W, W.bz * W.bz)));
                }
        double h = vmin(vmin(p.dx(), p.dy()), p.dz());
        double dt_h = p.cfl * h / maxs;
        double dt_r = 1e100;
        if (p.eta > 0.0) dt_r = 0.25 * h * h / p.eta;
        return vmin(dt_h, dt_r);
    }

    // the main()'s snapshot store (M3:1293-1321): out[0..10] = rho, P, Mach,
    // u, v, w, vabs, Bx, By, Bz, divB per cell
    void derived(const M3State<T>& s, double* const* out) const {
        for (int k = 0; k < p.nz; k++)
            for (int j = 0; j < p.ny; j++)
                for (int i = 0; i < p.nx; i++) {
                    const size_t q = cid(i, j, k);
                    const Prim8<T> W = to_prim(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc(s, i, j, k),
                                               by_cc(s, i, j, k), bz_cc(s, i, j, k));
                    const T cs = osqrt(a2(W));
                    const T vabs = osqrt(W.u * W.u + W.v * W.v + W.w * W.w);
                    const T mach = vabs / vmax(cs, T(1e-12));
                    const double d = ((double)bxf(s, i + 1, j, k) - (double)bxf(s, i, j, k)) / p.dx() +
                                     ((double)byf(s, i, j + 1, k) - (double)byf(s, i, j, k)) / p.dy() +
                                     ((double)bzf(s, i, j, k + 1) - (double)bzf(s, i, j, k)) / p.dz();
                    const double v[11] = {(double)W.r, (double)W.P, (double)mach, (double)W.u, (double)W.v,
                                          (double)W.w, (double)vabs, (double)W.bx, (double)W.by, (double)W.bz, d};
                    for (int m = 0; m < 11; m++) out[m][q] = v[m];
                }
    }

    double max_divB(const M3State<T>& s) const {  // M3:1070-1078
        double m = 0.0;
        for (int k = 0; k < p.nz; k++)
            for (int j = 0; j < p.ny; j++)
                for (int i = 0; i < p.nx; i++) {
                    double d = ((double)bxf(s, i + 1, j, k) - (double)bxf(s, i, j, k)) / p.dx() +
                               ((double)byf(s, i, j + 1, k) - (double)byf(s, i, j, k)) / p.dy() +
                               ((double)bzf(s, i, j, k + 1) - (double)bzf(s, i, j, k)) / p.dz();
                    m = vmax(m, std::abs(d));
                }
        return m;
    }
};

}  // namespace cco
