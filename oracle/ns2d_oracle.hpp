// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// CPU restatement of the 2D compressible Navier-Stokes + self-gravity step of
// navier_stokes_2d_hllc_poisson.cpp (cited NS:<line>): cons_to_prim, the
// first-order HLLC of the two cells beside each face (star energy with the
// star pressure), the explicit viscous stress flux from face-averaged centred
// velocity gradients, the gravity source from a periodic potential, and the
// Heun (SSP-RK2) loop body of main().  Periodic in x and y.  The potential is
// supplied by the caller (the spectral solve of poisson_oracle.hpp).
#pragma once
#include <cmath>
#include <functional>
#include <random>
#include <vector>

#include "oracle_common.hpp"

namespace cco {

struct NSPar {
    double gamma, cfl, x0, x1, y0, y1;
    int nx, ny;
    double floor_rho, floor_P;
    bool viscosity;
    double mu, cfl_visc;
    bool gravity;
    double G;
    double dx() const { return (x1 - x0) / nx; }   // Grid2D (NS:95-111)
    double dy() const { return (y1 - y0) / ny; }
};

template <class T> struct NSState { std::vector<T> d, mx, my, E; };

template <class T> class NS {
public:
    struct Prim { T d, u, v, P; };
    struct Flux { T f[4]; };   // {mass, x-momentum, y-momentum, energy}
    NSPar p;
    T gm1, idx1, idy1, idx2, idy2;
    explicit NS(const NSPar& par) : p(par) {
        gm1 = T(par.gamma - 1.0);
        idx1 = T(1.0 / par.dx()); idy1 = T(1.0 / par.dy());
        idx2 = T(1.0 / (2.0 * par.dx())); idy2 = T(1.0 / (2.0 * par.dy()));
    }
    int at(int i, int j) const { return wrap(i, p.nx) + p.nx * wrap(j, p.ny); }
    static int wrap(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }   // imod (NS:113-116)

    Prim prim(T d, T mx, T my, T E) const {   // cons_to_prim (NS:119-132)
        Prim W;
        W.d = vmax(d, T(p.floor_rho));
        W.u = mx / W.d;
        W.v = my / W.d;
        const T ke = T(0.5) * W.d * (W.u * W.u + W.v * W.v);
        W.P = vmax(gm1 * (E - ke), T(p.floor_P));
        return W;
    }
    T sound(const Prim& W) const { return std::sqrt(T(p.gamma) * W.P / vmax(W.d, T(p.floor_rho))); }   // NS:147-149

    // HLLC across a face whose normal velocity is n and tangential t (hllc_x,
    // NS:212-269; hllc_y, NS:271-282, is this with u and v exchanged).
    // Returns {mass, normal momentum, tangential momentum, energy}.
    Flux hllc(T dL, T nL, T tL, T pL, T dR, T nR, T tR, T pR) const {
        const T g = T(p.gamma);
        const T aL = std::sqrt(g * pL / vmax(dL, T(p.floor_rho)));
        const T aR = std::sqrt(g * pR / vmax(dR, T(p.floor_rho)));
        const T EL = pL / gm1 + T(0.5) * dL * (nL * nL + tL * tL);
        const T ER = pR / gm1 + T(0.5) * dR * (nR * nR + tR * tR);
        const T SL = vmin(nL - aL, nR - aR), SR = vmax(nL + aL, nR + aR);
        const T num = (pR - pL) + dL * nL * (SL - nL) - dR * nR * (SR - nR);
        const T den = dL * (SL - nL) - dR * (SR - nR);
        const T SM = (std::abs(den) > T(0.0)) ? num / den : T(0.0);
        auto phys = [&](T d, T n, T t, T P) {   // flux_x_from_prim (NS:198-210)
            const T E = P / gm1 + T(0.5) * d * (n * n + t * t);
            Flux F;
            F.f[0] = d * n; F.f[1] = d * n * n + P; F.f[2] = d * n * t; F.f[3] = (E + P) * n;
            return F;
        };
        const Flux FL = phys(dL, nL, tL, pL), FR = phys(dR, nR, tR, pR);
        if (T(0.0) <= SL) return FL;
        if (T(0.0) >= SR) return FR;
        auto star = [&](const Flux& F0, T S, T d, T n, T t, T P, T E) {   // NS:235-268
            const T fac = d * (S - n) / (S - SM);
            const T pstar = P + d * (S - n) * (SM - n);
            const T Es = ((S - n) * E - P * n + pstar * SM) / (S - SM);
            Flux F;
            F.f[0] = F0.f[0] + S * (fac - d);
            F.f[1] = F0.f[1] + S * (fac * SM - d * n);
            F.f[2] = F0.f[2] + S * (fac * t - d * t);
            F.f[3] = F0.f[3] + S * (Es - E);
            return F;
        };
        return (T(0.0) < SM) ? star(FL, SL, dL, nL, tL, pL, EL) : star(FR, SR, dR, nR, tR, pR, ER);
    }

    // g = -grad phi by centred differences times 1/(2h) (compute_gravity_accel, NS:330-360)
    void gravity_accel(const std::vector<T>& phi, std::vector<T>& gx, std::vector<T>& gy) const {
        const int nx = p.nx, ny = p.ny;
        gx.assign((size_t)nx * ny, T(0));
        gy.assign((size_t)nx * ny, T(0));
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                gx[at(i, j)] = -(phi[at(i + 1, j)] - phi[at(i - 1, j)]) * idx2;
                gy[at(i, j)] = -(phi[at(i, j + 1)] - phi[at(i, j - 1)]) * idy2;
            }
    }

    std::vector<Prim> prims(const NSState<T>& s) const {
        std::vector<Prim> W(s.d.size());
        for (size_t q = 0; q < W.size(); q++) W[q] = prim(s.d[q], s.mx[q], s.my[q], s.E[q]);
        return W;
    }

    // potential of a (floored) density field, the Poisson solve of the rhs (NS:379-383)
    using Potential = std::function<void(const std::vector<T>& rho, std::vector<T>& phi)>;

    // compute_rhs (NS:363-518).  X[q]: the face between cell q = (i, j) and
    // (i+1, j); Y[q]: between (i, j) and (i, j+1).
    NSState<T> rhs(const NSState<T>& s, const Potential& pot) const {
        const int nx = p.nx, ny = p.ny;
        const size_t N = (size_t)nx * ny;
        const std::vector<Prim> W = prims(s);
        std::vector<T> gx, gy;
        if (p.gravity) {
            std::vector<T> rho(N), phi;
            for (size_t q = 0; q < N; q++) rho[q] = W[q].d;
            pot(rho, phi);
            gravity_accel(phi, gx, gy);
        }
        std::vector<Flux> X(N), Y(N);
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const Prim& L = W[at(i, j)];
                const Prim& R = W[at(i + 1, j)];
                X[at(i, j)] = hllc(L.d, L.u, L.v, L.P, R.d, R.u, R.v, R.P);
                const Prim& B = W[at(i, j + 1)];
                const Flux F = hllc(L.d, L.v, L.u, L.P, B.d, B.v, B.u, B.P);
                Flux G;
                G.f[0] = F.f[0]; G.f[1] = F.f[2]; G.f[2] = F.f[1]; G.f[3] = F.f[3];
                Y[at(i, j)] = G;
            }
        if (p.viscosity && p.mu > 0.0) {   // NS:400-481
            std::vector<T> ux(N), uy(N), vx(N), vy(N);
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    const int q = at(i, j);
                    ux[q] = (W[at(i + 1, j)].u - W[at(i - 1, j)].u) * idx2;
                    vx[q] = (W[at(i + 1, j)].v - W[at(i - 1, j)].v) * idx2;
                    uy[q] = (W[at(i, j + 1)].u - W[at(i, j - 1)].u) * idy2;
                    vy[q] = (W[at(i, j + 1)].v - W[at(i, j - 1)].v) * idy2;
                }
            const T mu = T(p.mu), half = T(0.5), two = T(2.0), c23 = T(2.0) / T(3.0);
            for (int j = 0; j < ny; j++)
                for (int i = 0; i < nx; i++) {
                    for (int dir = 0; dir < 2; dir++) {
                        const int a = at(i, j), b = dir == 0 ? at(i + 1, j) : at(i, j + 1);
                        const T dudx = half * (ux[a] + ux[b]), dudy = half * (uy[a] + uy[b]);
                        const T dvdx = half * (vx[a] + vx[b]), dvdy = half * (vy[a] + vy[b]);
                        const T divv = dudx + dvdy;
                        const T tau_xy = mu * (dudy + dvdx);
                        const T uf = half * (W[a].u + W[b].u), vf = half * (W[a].v + W[b].v);
                        if (dir == 0) {
                            const T tau_xx = mu * (two * dudx - c23 * divv);
                            Flux& F = X[a];
                            F.f[1] += -tau_xx;
                            F.f[2] += -tau_xy;
                            F.f[3] += -(uf * tau_xx + vf * tau_xy);
                        } else {
                            const T tau_yy = mu * (two * dvdy - c23 * divv);
                            Flux& F = Y[a];
                            F.f[1] += -tau_xy;
                            F.f[2] += -tau_yy;
                            F.f[3] += -(uf * tau_xy + vf * tau_yy);
                        }
                    }
                }
        }
        NSState<T> d;
        d.d.resize(N); d.mx.resize(N); d.my.resize(N); d.E.resize(N);
        std::vector<T>* out[4] = {&d.d, &d.mx, &d.my, &d.E};
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) {
                const int q = at(i, j), qw = at(i - 1, j), qs = at(i, j - 1);
                T R[4];
                for (int m = 0; m < 4; m++)
                    R[m] = -(X[q].f[m] - X[qw].f[m]) * idx1 - (Y[q].f[m] - Y[qs].f[m]) * idy1;
                if (p.gravity) {
                    R[1] += W[q].d * gx[q];
                    R[2] += W[q].d * gy[q];
                    R[3] += W[q].d * (W[q].u * gx[q] + W[q].v * gy[q]);
                }
                for (int m = 0; m < 4; m++) (*out[m])[q] = R[m];
            }
        return d;
    }

    // the main() loop's Heun step (NS:762-781)
    void heun(NSState<T>& U, T dt, const Potential& pot) const {
        const size_t N = U.d.size();
        const T floor_rho = T(p.floor_rho);
        const NSState<T> k1 = rhs(U, pot);
        NSState<T> U1 = U;
        for (size_t q = 0; q < N; q++) {
            U1.d[q] = U.d[q] + dt * k1.d[q];
            U1.mx[q] = U.mx[q] + dt * k1.mx[q];
            U1.my[q] = U.my[q] + dt * k1.my[q];
            U1.E[q] = U.E[q] + dt * k1.E[q];
            if (U1.d[q] < floor_rho) U1.d[q] = floor_rho;
        }
        const NSState<T> k2 = rhs(U1, pot);
        const T h = T(0.5) * dt;
        for (size_t q = 0; q < N; q++) {
            U.d[q] = U.d[q] + h * (k1.d[q] + k2.d[q]);
            U.mx[q] = U.mx[q] + h * (k1.mx[q] + k2.mx[q]);
            U.my[q] = U.my[q] + h * (k1.my[q] + k2.my[q]);
            U.E[q] = U.E[q] + h * (k1.E[q] + k2.E[q]);
            if (U.d[q] < floor_rho) U.d[q] = floor_rho;
        }
    }

    // compute_dt (NS:521-546); per-cell speeds in T, the extrema and dt in double
    double compute_dt(const NSState<T>& s) const {
        double smax = 0.0, rho_min = 1e300;
        for (size_t q = 0; q < s.d.size(); q++) {
            const Prim W = prim(s.d[q], s.mx[q], s.my[q], s.E[q]);
            const T a = sound(W);
            smax = vmax(smax, (double)(std::abs(W.u) + a));
            smax = vmax(smax, (double)(std::abs(W.v) + a));
            rho_min = vmin(rho_min, (double)W.d);
        }
        const double h = vmin(p.dx(), p.dy());
        const double dt_hyp = (smax > 0.0) ? (p.cfl * h / smax) : 1e-6;
        double dt = dt_hyp;
        if (p.viscosity && p.mu > 0.0) {
            const double nu_max = p.mu / vmax(rho_min, p.floor_rho);
            const double dt_visc = (nu_max > 0.0) ? (p.cfl_visc * h * h / nu_max) : dt_hyp;
            dt = vmin(dt, dt_visc);
        }
        return dt;
    }

    // the store's fields (NS:698-746): rho, P, Mach, u, v, momx, momy, Phi
    void derived(const NSState<T>& s, const Potential& pot, double* const* out) const {
        const size_t N = s.d.size();
        std::vector<T> rho(N), phi(N, T(0));
        for (size_t q = 0; q < N; q++) {
            const Prim W = prim(s.d[q], s.mx[q], s.my[q], s.E[q]);
            const T a = sound(W);
            const T vmag = std::sqrt(W.u * W.u + W.v * W.v);
            rho[q] = W.d;
            const double v[7] = {(double)W.d, (double)W.P, (double)((a > T(0.0)) ? (vmag / a) : T(0.0)),
                                 (double)W.u, (double)W.v, (double)(W.d * W.u), (double)(W.d * W.v)};
            for (int m = 0; m < 7; m++)
                if (out[m]) out[m][q] = v[m];
        }
        if (p.gravity) pot(rho, phi);
        if (out[7])
            for (size_t q = 0; q < N; q++) out[7][q] = (double)phi[q];
    }
};

// the collapse IC of the reference main() (NS:627-689): mt19937(seed) and
// normal_distribution<double>(0, 1); per cell one density-noise draw, then u, v
inline void ns_ic_collapse(const NSPar& p, unsigned seed, NSState<double>& s) {
    const int nx = p.nx, ny = p.ny;
    const size_t N = (size_t)nx * ny;
    s.d.resize(N); s.mx.resize(N); s.my.resize(N); s.E.resize(N);
    std::mt19937 rng(seed);
    std::normal_distribution<double> gauss(0.0, 1.0);
    const double Lx = p.x1 - p.x0, Ly = p.y1 - p.y0;
    const double sigma = 0.10 * vmin(Lx, Ly);
    const double a0 = std::sqrt(p.gamma * 0.05 / 1.0), vamp = 0.05 * a0;
    const double xc = 0.5 * (p.x0 + p.x1), yc = 0.5 * (p.y0 + p.y1);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const double rx = (p.x0 + (i + 0.5) * p.dx()) - xc, ry = (p.y0 + (j + 0.5) * p.dy()) - yc;
            const double r2 = rx * rx + ry * ry;
            const double bump = 1.0 * std::exp(-0.5 * r2 / (sigma * sigma));
            const double noise = 0.01 * gauss(rng);
            const double rho = vmax(1.0 * (1.0 + bump + noise), p.floor_rho);
            const double P = vmax(0.05, p.floor_P);
            const double u = vamp * gauss(rng), v = vamp * gauss(rng);
            const double d = vmax(rho, p.floor_rho), Pc = vmax(P, p.floor_P);   // prim_to_cons (NS:134-145)
            const size_t q = (size_t)j * nx + i;
            s.d[q] = d; s.mx[q] = d * u; s.my[q] = d * v;
            s.E[q] = Pc / (p.gamma - 1.0) + 0.5 * d * (u * u + v * v);
        }
}

}  // namespace cco
