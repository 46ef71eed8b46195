// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// CPU restatement of the 2D Euler + self-gravity step of euler2d_gravity_hllc.cpp
// (cited EH:<line>): MUSCL-MC on primitives with a 4-point stencil per face,
// the reference HLLC (star energy with P, not P*), gravity inside the
// right-hand side, SSP-RK2.  The Poisson solve is supplied by the caller.
#pragma once
#include <array>
#include <cmath>
#include <vector>

#include "oracle_common.hpp"

namespace cco {

struct EHPar {
    double gamma, cfl, x0, x1, y0, y1;
    int nx, ny;
    double floor_rho, floor_P;
    bool px, py;
    bool gravity;
    double dx() const { return (x1 - x0) / nx; }
    double dy() const { return (y1 - y0) / ny; }
};

template <class T> struct EHState { std::vector<T> rho, mx, my, E; };
template <class T> struct EPrim { T r, u, v, P; };
template <class T> struct EFlux { T f[4]; };

template <class T> class EH {
public:
    EHPar p;
    Axis ax, ay;
    T gm1;
    explicit EH(const EHPar& par) : p(par), ax{par.nx, par.px}, ay{par.ny, par.py}, gm1(T(par.gamma) - T(1.0)) {}

    void floors(T& rho, T& mx, T& my, T& E) const {  // EH:62-72
        rho = vmax(rho, T(p.floor_rho));
        T u = mx / rho, v = my / rho;
        T kin = T(0.5) * rho * (u * u + v * v);
        T P = gm1 * (E - kin);
        if (P < T(p.floor_P)) {
            T eint = T(p.floor_P) / gm1;
            E = kin + eint;
        }
    }
    // cons_to_prim_full (EH:74-83) -> (u, v, P, a); cons_to_prim (EH:96-100)
    EPrim<T> to_prim(T rho, T mx, T my, T E, T* a_out = nullptr) const {
        T r = vmax(rho, T(p.floor_rho));
        T u = mx / r, v = my / r;
        T kin = T(0.5) * r * (u * u + v * v);
        T P = gm1 * (E - kin);
        if (P < T(p.floor_P)) P = T(p.floor_P);
        if (a_out) *a_out = std::sqrt(T(p.gamma) * P / r);
        return {vmax(rho, T(p.floor_rho)), u, v, P};
    }
    // the main()'s snapshot store (EH:661-689): out = rho, P, Mach per cell
    void derived(const EHState<T>& s, double* const* out) const {
        const size_t n = (size_t)p.nx * p.ny;
        for (size_t q = 0; q < n; q++) {
            T rho = s.rho[q], mx = s.mx[q], my = s.my[q], E = s.E[q];
            floors(rho, mx, my, E);
            T a;
            const EPrim<T> W = to_prim(rho, mx, my, E, &a);
            const T vmag = std::sqrt(W.u * W.u + W.v * W.v);
            out[0][q] = (double)rho;
            out[1][q] = (double)W.P;
            out[2][q] = (a > T(0.0)) ? (double)(vmag / a) : 0.0;
        }
    }
    // prim_to_cons (EH:102-109)
    void to_cons(const EPrim<T>& W, T& r, T& mx, T& my, T& E) const {
        r = vmax(W.r, T(p.floor_rho));
        mx = r * W.u;
        my = r * W.v;
        T kin = T(0.5) * r * (W.u * W.u + W.v * W.v);
        T eint = W.P / gm1;
        E = kin + eint;
    }
    // HLLC along x (dir 0) or y (dir 1) (EH:125-219); n = normal velocity
    EFlux<T> hllc(const EPrim<T>& WL, const EPrim<T>& WR, int dir) const {
        const T g = T(p.gamma);
        T aL = std::sqrt(g * WL.P / vmax(WL.r, T(p.floor_rho)));
        T aR = std::sqrt(g * WR.P / vmax(WR.r, T(p.floor_rho)));
        T nL = dir == 0 ? WL.u : WL.v, nR = dir == 0 ? WR.u : WR.v;
        T SL = vmin(nL - aL, nR - aR);
        T SR = vmax(nL + aL, nR + aR);
        T rL, mLx, mLy, EL, rR, mRx, mRy, ER;
        to_cons(WL, rL, mLx, mLy, EL);
        to_cons(WR, rR, mRx, mRy, ER);
        auto flux = [&](const EPrim<T>& W) {  // euler_flux_x / euler_flux_y (EH:113-123)
            T E = W.P / gm1 + T(0.5) * W.r * (W.u * W.u + W.v * W.v);
            EFlux<T> F;
            if (dir == 0) { F.f[0] = W.r * W.u; F.f[1] = W.r * W.u * W.u + W.P; F.f[2] = W.r * W.u * W.v; F.f[3] = (E + W.P) * W.u; }
            else          { F.f[0] = W.r * W.v; F.f[1] = W.r * W.u * W.v; F.f[2] = W.r * W.v * W.v + W.P; F.f[3] = (E + W.P) * W.v; }
            return F;
        };
        EFlux<T> FL = flux(WL), FR = flux(WR);
        T num = (WR.P - WL.P) + rL * nL * (SL - nL) - rR * nR * (SR - nR);
        T den = rL * (SL - nL) - rR * (SR - nR);
        T SM = (std::abs(den) > T(1e-14)) ? (num / den) : T(0.0);
        if (T(0.0) <= SL) return FL;
        if (T(0.0) >= SR) return FR;
        auto star = [&](const EPrim<T>& W, T r, T E, T S) {
            T n = dir == 0 ? W.u : W.v, t = dir == 0 ? W.v : W.u;
            T rS = r * (S - n) / (S - SM);
            T mn = rS * SM, mt = rS * t;
            T ES = ((S - n) * E - W.P * n + W.P * SM) / (S - SM);
            return dir == 0 ? std::array<T, 4>{rS, mn, mt, ES} : std::array<T, 4>{rS, mt, mn, ES};
        };
        EFlux<T> F;
        if (T(0.0) < SM) {
            auto Us = star(WL, rL, EL, SL);
            T U0[4] = {rL, mLx, mLy, EL};
            for (int k = 0; k < 4; k++) F.f[k] = FL.f[k] + SL * (Us[k] - U0[k]);
        } else {
            auto Us = star(WR, rR, ER, SR);
            T U0[4] = {rR, mRx, mRy, ER};
            for (int k = 0; k < 4; k++) F.f[k] = FR.f[k] + SR * (Us[k] - U0[k]);
        }
        return F;
    }

    // rhs (EH:406-527); gx, gy supplied (the reference computes them inside, EH:411)
    EHState<T> rhs(const EHState<T>& U, const std::vector<T>& gx, const std::vector<T>& gy) const {
        const int nx = p.nx, ny = p.ny;
        const T dx = T(p.dx()), dy = T(p.dy());
        const size_t N = (size_t)nx * ny;
        EHState<T> d;
        d.rho.assign(N, T(0)); d.mx.assign(N, T(0)); d.my.assign(N, T(0)); d.E.assign(N, T(0));
        std::vector<EPrim<T>> W(N);
        for (size_t k = 0; k < N; k++) {
            T r = U.rho[k], mx = U.mx[k], my = U.my[k], E = U.E[k];
            floors(r, mx, my, E);
            W[k] = to_prim(r, mx, my, E);
        }
        auto face = [&](const EPrim<T>& wm, const EPrim<T>& w0, const EPrim<T>& wp, const EPrim<T>& wpp,
                        EPrim<T>& L, EPrim<T>& R) {
            auto lr = [&](T a, T b, T c, T e, T& l, T& r) {
                T sL = mc_slope(b - a, c - b), sR = mc_slope(c - b, e - c);
                l = b + T(0.5) * sL;
                r = c - T(0.5) * sR;
            };
            lr(wm.r, w0.r, wp.r, wpp.r, L.r, R.r);
            lr(wm.u, w0.u, wp.u, wpp.u, L.u, R.u);
            lr(wm.v, w0.v, wp.v, wpp.v, L.v, R.v);
            lr(wm.P, w0.P, wp.P, wpp.P, L.P, R.P);
            L.r = vmax(L.r, T(p.floor_rho)); R.r = vmax(R.r, T(p.floor_rho));
            L.P = vmax(L.P, T(p.floor_P));   R.P = vmax(R.P, T(p.floor_P));
        };
        std::vector<EFlux<T>> Fx((size_t)(nx + 1) * ny), Fy((size_t)nx * (ny + 1));
        for (int j = 0; j < ny; j++)
            for (int i = 0; i <= nx; i++) {
                int iL = ax.cell(i - 1), iR = ax.cell(i);
                auto at = [&](int ii) { return W[(size_t)j * nx + ax.cell(ii)]; };
                EPrim<T> L, R;
                face(at(iL - 1), at(iL), at(iR), at(iR + 1), L, R);
                Fx[(size_t)j * (nx + 1) + i] = hllc(L, R, 0);
            }
        for (int j = 0; j <= ny; j++)
            for (int i = 0; i < nx; i++) {
                int jL = ay.cell(j - 1), jR = ay.cell(j);
                auto at = [&](int jj) { return W[(size_t)ay.cell(jj) * nx + i]; };
                EPrim<T> L, R;
                face(at(jL - 1), at(jL), at(jR), at(jR + 1), L, R);
                Fy[(size_t)j * nx + i] = hllc(L, R, 1);
            }
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                size_t k = (size_t)j * nx + i;
                const EFlux<T>&R = Fx[(size_t)j * (nx + 1) + i + 1], &L = Fx[(size_t)j * (nx + 1) + i];
                const EFlux<T>&Uf = Fy[(size_t)(j + 1) * nx + i], &D = Fy[(size_t)j * nx + i];
                d.rho[k] = -(R.f[0] - L.f[0]) / dx - (Uf.f[0] - D.f[0]) / dy;
                d.mx[k] = -(R.f[1] - L.f[1]) / dx - (Uf.f[1] - D.f[1]) / dy;
                d.my[k] = -(R.f[2] - L.f[2]) / dx - (Uf.f[2] - D.f[2]) / dy;
                d.E[k] = -(R.f[3] - L.f[3]) / dx - (Uf.f[3] - D.f[3]) / dy;
                if (p.gravity) {
                    T rho = vmax(U.rho[k], T(p.floor_rho));
                    T u = U.mx[k] / rho, v = U.my[k] / rho;
                    d.mx[k] += rho * gx[k];
                    d.my[k] += rho * gy[k];
                    d.E[k] += rho * (u * gx[k] + v * gy[k]);
                }
            }
        return d;
    }

    // rk2_step (EH:529-550); grav(U, gx, gy) computes the gravity of a state
    template <class GravFn> void rk2_step(EHState<T>& U, T dt, GravFn grav) const {
        std::vector<T> gx, gy;
        grav(U, gx, gy);
        EHState<T> k1 = rhs(U, gx, gy);
        EHState<T> U1 = U;
        const size_t N = U.rho.size();
        for (size_t q = 0; q < N; q++) {
            U1.rho[q] += dt * k1.rho[q];
            U1.mx[q] += dt * k1.mx[q];
            U1.my[q] += dt * k1.my[q];
            U1.E[q] += dt * k1.E[q];
            floors(U1.rho[q], U1.mx[q], U1.my[q], U1.E[q]);
        }
        grav(U1, gx, gy);
        EHState<T> k2 = rhs(U1, gx, gy);
        for (size_t q = 0; q < N; q++) {
            U.rho[q] = T(0.5) * U.rho[q] + T(0.5) * (U1.rho[q] + dt * k2.rho[q]);
            U.mx[q] = T(0.5) * U.mx[q] + T(0.5) * (U1.mx[q] + dt * k2.mx[q]);
            U.my[q] = T(0.5) * U.my[q] + T(0.5) * (U1.my[q] + dt * k2.my[q]);
            U.E[q] = T(0.5) * U.E[q] + T(0.5) * (U1.E[q] + dt * k2.E[q]);
            floors(U.rho[q], U.mx[q], U.my[q], U.E[q]);
        }
    }

    double compute_dt(const EHState<T>& U) const {  // EH:390-404
        double ms = 1e-30;
        for (size_t k = 0; k < U.rho.size(); k++) {
            T a;
            EPrim<T> W = to_prim(U.rho[k], U.mx[k], U.my[k], U.E[k], &a);
            ms = vmax(ms, (double)(std::abs(W.u) + a));
            ms = vmax(ms, (double)(std::abs(W.v) + a));
        }
        return p.cfl * vmin(p.dx(), p.dy()) / ms;
    }
};

}  // namespace cco
