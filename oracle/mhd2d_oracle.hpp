// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// CPU restatement of the 2D resistive-MHD + self-gravity step of
// mhd2d_resistive_hlld_ct_gravity.cpp (cited as M2:<line>).  Written for the
// tests: one pass per reference sub-step, plain loops, no fusion, so that each
// function can be read side by side with the reference line it restates.
#pragma once
#include <array>
#include <cmath>
#include <vector>

#include "oracle_common.hpp"

namespace cco {

struct M2Par {
    double gamma, cfl, x0, x1, y0, y1;
    int nx, ny;
    double floor_rho, floor_P;
    bool px, py;
    double eta;
    bool gravity;
    double G;
    int sor_iters;
    double sor_omega, sor_tol;
    double dx() const { return (x1 - x0) / nx; }
    double dy() const { return (y1 - y0) / ny; }
};

template <class T> struct M2State {
    std::vector<T> rho, mx, my, mz, E, Bz;  // cells, q = j*nx+i
    std::vector<T> bxf;                     // (nx+1)*ny, j*(nx+1)+i_face
    std::vector<T> byf;                     // nx*(ny+1), j_face*nx+i
};

template <class T> class M2 {
public:
    M2Par p;
    Axis ax, ay;
    T gm1;
    explicit M2(const M2Par& par) : p(par), ax{par.nx, par.px}, ay{par.ny, par.py}, gm1(T(par.gamma) - T(1.0)) {}

    size_t cidx(int i, int j) const { return (size_t)ay.cell(j) * p.nx + ax.cell(i); }
    // face lookups with the reference's wrap rules (M2:241-252)
    T bx_face(const M2State<T>& s, int i_face, int j) const {
        return s.bxf[(size_t)ay.cell(j) * (p.nx + 1) + ax.face(i_face)];
    }
    T by_face(const M2State<T>& s, int i, int j_face) const {
        return s.byf[(size_t)ay.face(j_face) * p.nx + ax.cell(i)];
    }
    // cell-centred in-plane B from the two faces (M2:254-276)
    T bx_cc(const M2State<T>& s, int i, int j) const {
        return T(0.5) * (bx_face(s, i, j) + bx_face(s, i + 1, j));
    }
    T by_cc(const M2State<T>& s, int i, int j) const {
        return T(0.5) * (by_face(s, i, j) + by_face(s, i, j + 1));
    }

    // enforce_floors (M2:114-124)
    void floors(T& rho, T& mx, T& my, T& mz, T& E, T Bx, T By, T Bz) const {
        rho = vmax(rho, T(p.floor_rho));
        T u = mx / rho, v = my / rho, w = mz / rho;
        T kin = T(0.5) * rho * (u * u + v * v + w * w);
        T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
        T P = gm1 * (E - kin - mag);
        if (P < T(p.floor_P)) {
            T eint = T(p.floor_P) / gm1;
            E = kin + mag + eint;
        }
    }
    // cons_to_prim (M2:126-135)
    Prim8<T> to_prim(T rho, T mx, T my, T mz, T E, T Bx, T By, T Bz) const {
        rho = vmax(rho, T(p.floor_rho));
        T u = mx / rho, v = my / rho, w = mz / rho;
        T kin = T(0.5) * rho * (u * u + v * v + w * w);
        T mag = T(0.5) * (Bx * Bx + By * By + Bz * Bz);
        T P = gm1 * (E - kin - mag);
        if (P < T(p.floor_P)) P = T(p.floor_P);
        return {rho, u, v, w, P, Bx, By, Bz};
    }
    // get_prim_cc (M2:278-286): wrap first, then use the wrapped cell's faces
    Prim8<T> prim_at(const M2State<T>& s, int i, int j) const {
        int ii = ax.cell(i), jj = ay.cell(j);
        size_t q = (size_t)jj * p.nx + ii;
        return to_prim(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc(s, ii, jj), by_cc(s, ii, jj), s.Bz[q]);
    }
    // ideal-gas energy of a primitive state (M2:357, 397, 482, 495)
    T energy(const Prim8<T>& W) const {
        T B2 = W.bx * W.bx + W.by * W.by + W.bz * W.bz;
        return W.P / gm1 + T(0.5) * W.r * (W.u * W.u + W.v * W.v + W.w * W.w) + T(0.5) * B2;
    }
    // fast magnetosonic speed along the component bn2 = Bn*Bn (M2:148-174)
    T fast(const Prim8<T>& W, T bn2) const {
        T a2 = T(p.gamma) * W.P / vmax(W.r, T(p.floor_rho));
        T b2 = W.bx * W.bx + W.by * W.by + W.bz * W.bz;
        T rho = vmax(W.r, T(1e-300));
        T vA2 = b2 / rho;
        T vn2 = bn2 / rho;
        T disc = (a2 + vA2) * (a2 + vA2) - T(4.0) * a2 * vn2;
        disc = vmax(T(0.0), disc);
        T cf2 = T(0.5) * ((a2 + vA2) + osqrt(disc));
        return osqrt(vmax(T(0.0), cf2));
    }

    // x-normal ideal flux (M2:351-370) and HLLD (M2:372-530)
    Flux7<T> flux_x(const Prim8<T>& W) const { return ideal_flux_x(*this, W); }
    Flux7<T> hlld_x(Prim8<T> L, Prim8<T> R, T Bn) const { return hlld_x_generic(*this, L, R, Bn); }

    // y-normal HLLD by the (u,v)/(Bx,By) swap (M2:540-561); output
    // f[1]=flux of mx, f[2]=flux of my, f[5]=flux of Bx, f[6]=flux of Bz
    Flux7<T> hlld_y(Prim8<T> L, Prim8<T> R, T Bn) const {
        L.by = Bn; R.by = Bn;
        Prim8<T> aL{L.r, L.v, L.u, L.w, L.P, L.by, L.bx, L.bz};
        Prim8<T> aR{R.r, R.v, R.u, R.w, R.P, R.by, R.bx, R.bz};
        Flux7<T> Fx = hlld_x(aL, aR, Bn);
        Flux7<T> G = Fx;
        G.f[1] = Fx.f[2];
        G.f[2] = Fx.f[1];
        return G;
    }

    // MUSCL-MC face states of one cell (M2:290-336).  dir 0: x, 1: y.
    void recon(const M2State<T>& s, int i, int j, int dir, Prim8<T>& WL, Prim8<T>& WR) const {
        int di = dir == 0 ? 1 : 0, dj = dir == 0 ? 0 : 1;
        Prim8<T> Wm = prim_at(s, i - di, j - dj), Wc = prim_at(s, i, j), Wp = prim_at(s, i + di, j + dj);
        auto lim = [&](T wm, T wc, T wp) { return mc_slope(wc - wm, wp - wc); };
        T sr = lim(Wm.r, Wc.r, Wp.r), su = lim(Wm.u, Wc.u, Wp.u), sv = lim(Wm.v, Wc.v, Wp.v);
        T sw = lim(Wm.w, Wc.w, Wp.w), sP = lim(Wm.P, Wc.P, Wp.P);
        T st = dir == 0 ? lim(Wm.by, Wc.by, Wp.by) : lim(Wm.bx, Wc.bx, Wp.bx);
        T sz = lim(Wm.bz, Wc.bz, Wp.bz);
        WL = Wc; WR = Wc;
        WL.r = Wc.r - T(0.5) * sr; WR.r = Wc.r + T(0.5) * sr;
        WL.u = Wc.u - T(0.5) * su; WR.u = Wc.u + T(0.5) * su;
        WL.v = Wc.v - T(0.5) * sv; WR.v = Wc.v + T(0.5) * sv;
        WL.w = Wc.w - T(0.5) * sw; WR.w = Wc.w + T(0.5) * sw;
        WL.P = Wc.P - T(0.5) * sP; WR.P = Wc.P + T(0.5) * sP;
        if (dir == 0) { WL.by = Wc.by - T(0.5) * st; WR.by = Wc.by + T(0.5) * st; }
        else          { WL.bx = Wc.bx - T(0.5) * st; WR.bx = Wc.bx + T(0.5) * st; }
        WL.bz = Wc.bz - T(0.5) * sz; WR.bz = Wc.bz + T(0.5) * sz;
        WL.r = vmax(WL.r, T(p.floor_rho)); WR.r = vmax(WR.r, T(p.floor_rho));
        WL.P = vmax(WL.P, T(p.floor_P));   WR.P = vmax(WR.P, T(p.floor_P));
    }

    // advance_stage (M2:690-834): s0 -> s1 with gravity g (gx, gy per cell)
    void advance_stage(const M2State<T>& s0, M2State<T>& s1, const std::vector<T>& gx,
                       const std::vector<T>& gy, T dt) const {
        const int nx = p.nx, ny = p.ny;
        const T dx = T(p.dx()), dy = T(p.dy());
        s1 = s0;
        std::vector<Flux7<T>> Fx((size_t)(nx + 1) * ny), Gy((size_t)nx * (ny + 1));
        // x faces (M2:706-725)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i <= nx; i++) {
                Prim8<T> a, WL, WR, b;
                recon(s0, ax.cell(i - 1), j, 0, a, WL);
                recon(s0, ax.cell(i), j, 0, WR, b);
                Fx[(size_t)j * (nx + 1) + i] = hlld_x(WL, WR, bx_face(s0, i, j));
            }
        // y faces (M2:728-747)
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i < nx; i++) {
                Prim8<T> a, WL, WR, b;
                recon(s0, i, ay.cell(j - 1), 1, a, WL);
                recon(s0, i, ay.cell(j), 1, WR, b);
                Gy[(size_t)j * nx + i] = hlld_y(WL, WR, by_face(s0, i, j));
            }
        // FV update + floors with the stage-input B (M2:750-779)
        const T idx = T(1.0) / dx, idy = T(1.0) / dy;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t q = (size_t)j * nx + i;
                const Flux7<T>& R = Fx[(size_t)j * (nx + 1) + i + 1];
                const Flux7<T>& L = Fx[(size_t)j * (nx + 1) + i];
                const Flux7<T>& U = Gy[(size_t)(j + 1) * nx + i];
                const Flux7<T>& D = Gy[(size_t)j * nx + i];
                T d[7];
                for (int k = 0; k < 7; k++) d[k] = -(R.f[k] - L.f[k]) * idx - (U.f[k] - D.f[k]) * idy;
                s1.rho[q] += dt * d[0];
                s1.mx[q] += dt * d[1];
                s1.my[q] += dt * d[2];
                s1.mz[q] += dt * d[3];
                s1.E[q] += dt * d[4];
                s1.Bz[q] += dt * d[6];
                floors(s1.rho[q], s1.mx[q], s1.my[q], s1.mz[q], s1.E[q], bx_cc(s0, i, j), by_cc(s0, i, j), s1.Bz[q]);
            }
        // edge EMF: arithmetic average of the four face EMFs + eta*Jz (M2:782-804, 565-575)
        // x-face EMF is -F(By), y-face EMF is +G(Bx)
        auto ex = [&](int i, int j) { return -Fx[(size_t)ay.cell(j) * (nx + 1) + ax.face(i)].f[5]; };
        auto ey = [&](int i, int j) { return Gy[(size_t)ay.face(j) * nx + ax.cell(i)].f[5]; };
        std::vector<T> Ez((size_t)(nx + 1) * (ny + 1));
        for (int je = 0; je <= ny; je++)
            for (int ie = 0; ie <= nx; ie++) {
                T ideal = T(0.25) * (ex(ie, je - 1) + ex(ie, je) + ey(ie - 1, je) + ey(ie, je));
                T res = T(0.0);
                if (p.eta > 0.0) {
                    T dBydx = (by_face(s0, ie, je) - by_face(s0, ie - 1, je)) / dx;
                    T dBxdy = (bx_face(s0, ie, je) - bx_face(s0, ie, je - 1)) / dy;
                    res = T(p.eta) * (dBydx - dBxdy);
                }
                Ez[(size_t)je * (nx + 1) + ie] = ideal + res;
            }
        // CT (M2:807-830)
        for (int j = 0; j < ny; j++)
            for (int i = 0; i <= nx; i++) {
                int j0 = ay.face(j), j1 = ay.face(j + 1);
                T eU = Ez[(size_t)j1 * (nx + 1) + i], eD = Ez[(size_t)j0 * (nx + 1) + i];
                s1.bxf[(size_t)j * (nx + 1) + i] += -(dt / dy) * (eU - eD);
            }
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i < nx; i++) {
                int i0 = ax.face(i), i1 = ax.face(i + 1);
                T eR = Ez[(size_t)j * (nx + 1) + i1], eL = Ez[(size_t)j * (nx + 1) + i0];
                s1.byf[(size_t)j * nx + i] += +(dt / dx) * (eR - eL);
            }
        gravity_sources(s1, gx, gy, dt);
        joule_and_bz(s1, dt);
    }

    // add_gravity_sources (M2:602-629)
    void gravity_sources(M2State<T>& s, const std::vector<T>& gx, const std::vector<T>& gy, T dt) const {
        if (!p.gravity) return;
        const int nx = p.nx, ny = p.ny;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t q = (size_t)j * nx + i;
                T rho = s.rho[q], gxq = gx[q], gyq = gy[q];
                T u = s.mx[q] / vmax(rho, T(1e-300));
                T v = s.my[q] / vmax(rho, T(1e-300));
                s.mx[q] += dt * rho * gxq;
                s.my[q] += dt * rho * gyq;
                s.E[q] += dt * rho * (u * gxq + v * gyq);
            }
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t q = (size_t)j * nx + i;
                floors(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc(s, i, j), by_cc(s, i, j), s.Bz[q]);
            }
    }

    // add_joule_heating_and_Bz_resistive (M2:631-686)
    void joule_and_bz(M2State<T>& s, T dt) const {
        if (!(p.eta > 0.0)) return;
        const int nx = p.nx, ny = p.ny;
        const T dx = T(p.dx()), dy = T(p.dy()), eta = T(p.eta);
        auto bz = [&](int i, int j) { return s.Bz[cidx(i, j)]; };
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                T dBzdy = (bz(i, j + 1) - bz(i, j - 1)) / (T(2) * dy);
                T dBzdx = (bz(i + 1, j) - bz(i - 1, j)) / (T(2) * dx);
                T dBydx = (by_face(s, i + 1, j) - by_face(s, i, j)) / dx;
                T dBxdy = (bx_face(s, i, j + 1) - bx_face(s, i, j)) / dy;
                T Jx = dBzdy, Jy = -dBzdx, Jz = dBydx - dBxdy;
                T J2 = Jx * Jx + Jy * Jy + Jz * Jz;
                s.E[(size_t)j * nx + i] += dt * eta * J2;
            }
        std::vector<T> nb((size_t)nx * ny);
        const T idx2 = T(1.0) / (dx * dx), idy2 = T(1.0) / (dy * dy);
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                T lap = (bz(i + 1, j) - T(2) * bz(i, j) + bz(i - 1, j)) * idx2 +
                        (bz(i, j + 1) - T(2) * bz(i, j) + bz(i, j - 1)) * idy2;
                nb[(size_t)j * nx + i] = bz(i, j) + dt * eta * lap;
            }
        s.Bz.swap(nb);
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t q = (size_t)j * nx + i;
                floors(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc(s, i, j), by_cc(s, i, j), s.Bz[q]);
            }
    }

    // rk2_step (M2:838-869).  poisson(rho) -> (gx, gy) is the stage-2 solver.
    template <class PoissonFn>
    void rk2_step(M2State<T>& s, const std::vector<T>& gx, const std::vector<T>& gy, T dt, PoissonFn poisson) const {
        M2State<T> s1, s2;
        advance_stage(s, s1, gx, gy, dt);
        std::vector<T> g1x, g1y;
        poisson(s1.rho, g1x, g1y);
        advance_stage(s1, s2, g1x, g1y, dt);
        const size_t N = s.rho.size();
        for (size_t q = 0; q < N; q++) {
            s.rho[q] = T(0.5) * (s.rho[q] + s2.rho[q]);
            s.mx[q] = T(0.5) * (s.mx[q] + s2.mx[q]);
            s.my[q] = T(0.5) * (s.my[q] + s2.my[q]);
            s.mz[q] = T(0.5) * (s.mz[q] + s2.mz[q]);
            s.E[q] = T(0.5) * (s.E[q] + s2.E[q]);
            s.Bz[q] = T(0.5) * (s.Bz[q] + s2.Bz[q]);
        }
        for (size_t k = 0; k < s.bxf.size(); k++) s.bxf[k] = T(0.5) * (s.bxf[k] + s2.bxf[k]);
        for (size_t k = 0; k < s.byf.size(); k++) s.byf[k] = T(0.5) * (s.byf[k] + s2.byf[k]);
        for (int j = 0; j < p.ny; j++)
            for (int i = 0; i < p.nx; i++) {
                size_t q = (size_t)j * p.nx + i;
                floors(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], bx_cc(s, i, j), by_cc(s, i, j), s.Bz[q]);
            }
    }

    // compute_dt (M2:579-598), accumulated in double whatever T is
    double compute_dt(const M2State<T>& s) const {
        double maxs = 1e-14;
        for (int j = 0; j < p.ny; j++)
            for (int i = 0; i < p.nx; i++) {
                Prim8<T> W = prim_at(s, i, j);
                maxs = vmax(maxs, (double)(std::abs(W.u) + fast(W, W.bx * W.bx)));
                maxs = vmax(maxs, (double)(std::abs(W.v) + fast(W, W.by * W.by)));
            }
        double dxd = p.dx(), dyd = p.dy();
        double dt_h = p.cfl * vmin(dxd, dyd) / maxs;
        double dt_r = 1e100;
        if (p.eta > 0.0) {
            double h = vmin(dxd, dyd);
            dt_r = 0.25 * h * h / p.eta;
        }
        return vmin(dt_h, dt_r);
    }

    // the main()'s snapshot store (M2:1065-1106): out[0..9] = rho, P, Mach,
    // u, v, vabs, Bx_cc, By_cc, Bz, divB per cell
    void derived(const M2State<T>& s, double* const* out) const {
        const double dx = p.dx(), dy = p.dy();
        for (int j = 0; j < p.ny; j++)
            for (int i = 0; i < p.nx; i++) {
                const size_t q = (size_t)j * p.nx + i;
                const T Bx = bx_cc(s, i, j), By = by_cc(s, i, j);
                const Prim8<T> W = to_prim(s.rho[q], s.mx[q], s.my[q], s.mz[q], s.E[q], Bx, By, s.Bz[q]);
                const T cs = osqrt(vmax(T(0.0), T(p.gamma) * W.P / vmax(W.r, T(p.floor_rho))));
                const T vabs = osqrt(W.u * W.u + W.v * W.v + W.w * W.w);
                const T mach = vabs / vmax(cs, T(1e-14));
                const double d = ((double)bx_face(s, i + 1, j) - (double)bx_face(s, i, j)) / dx +
                                 ((double)by_face(s, i, j + 1) - (double)by_face(s, i, j)) / dy;
                const double v[10] = {(double)W.r, (double)W.P, (double)mach, (double)W.u, (double)W.v,
                                      (double)vabs, (double)Bx, (double)By, (double)W.bz, d};
                for (int k = 0; k < 10; k++) out[k][q] = v[k];
            }
    }

    // max |div B| per cell (M2:873-879)
    double max_divB(const M2State<T>& s) const {
        double m = 0.0, dx = p.dx(), dy = p.dy();
        for (int j = 0; j < p.ny; j++)
            for (int i = 0; i < p.nx; i++) {
                double d = ((double)bx_face(s, i + 1, j) - (double)bx_face(s, i, j)) / dx +
                           ((double)by_face(s, i, j + 1) - (double)by_face(s, i, j)) / dy;
                m = vmax(m, std::abs(d));
            }
        return m;
    }
};

}  // namespace cco
