// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// C ABI over the CPU restatements in this directory, for tests/ (through
// ctypes) and for bench.py's CPU-baseline leg.  Poisson ordering per call:
//   mode 0  lexicographic SOR, the reference's own ordering (M2:207-223, EH:335-368)
//   mode 1  red-black SOR, the ordering the GPU kernels use
//   mode 2  spectral FFT solve (NS:285-328)
//   mode 3  direct solve of the SOR's discrete problem, density mean in the
//           batched reduction order (the library's ensemble Poisson)
#include <cstring>
#include <algorithm>
#include <vector>

#include "../include/cc_step.h"
#include "mhd2d_oracle.hpp"
#include "mhd3d_oracle.hpp"
#include "euler2d_oracle.hpp"
#include "ns2d_oracle.hpp"
#include "poisson_oracle.hpp"

namespace {
using namespace cco;

M2Par m2par(const cc_mhd2d_params* c) {
    M2Par p;
    p.gamma = c->gamma; p.cfl = c->cfl;
    p.x0 = c->x0; p.x1 = c->x1; p.y0 = c->y0; p.y1 = c->y1;
    p.nx = c->Nx; p.ny = c->Ny;
    p.floor_rho = c->floor_rho; p.floor_P = c->floor_P;
    p.px = c->periodic_x != 0; p.py = c->periodic_y != 0;
    p.eta = c->eta; p.gravity = c->gravity_on != 0; p.G = c->G;
    p.sor_iters = c->sor_iters; p.sor_omega = c->sor_omega; p.sor_tol = c->sor_tol;
    return p;
}

PoissonSpec m2spec(const cc_mhd2d_params* c) {
    PoissonSpec s;
    s.nx = c->Nx; s.ny = c->Ny;
    s.px = c->periodic_x != 0; s.py = c->periodic_y != 0;
    s.dx = (c->x1 - c->x0) / c->Nx; s.dy = (c->y1 - c->y0) / c->Ny;
    s.G = c->G; s.omega = c->sor_omega; s.max_iter = c->sor_iters; s.tol = c->sor_tol;
    s.floor_density = false; s.floor_rho = c->floor_rho;
    s.Lx = c->x1 - c->x0; s.Ly = c->y1 - c->y0;
    return s;
}

template <class T> void load(const cc_mhd2d_params* c, const double* const* f, M2State<T>& s) {
    size_t N = (size_t)c->Nx * c->Ny, NX = (size_t)(c->Nx + 1) * c->Ny, NY = (size_t)c->Nx * (c->Ny + 1);
    std::vector<T>* cell[6] = {&s.rho, &s.mx, &s.my, &s.mz, &s.E, &s.Bz};
    for (int k = 0; k < 6; k++) cell[k]->assign(f[k], f[k] + N);
    s.bxf.assign(f[6], f[6] + NX);
    s.byf.assign(f[7], f[7] + NY);
}

template <class T> void store(const M2State<T>& s, double* const* f) {
    const std::vector<T>* v[8] = {&s.rho, &s.mx, &s.my, &s.mz, &s.E, &s.Bz, &s.bxf, &s.byf};
    for (int k = 0; k < 8; k++)
        for (size_t q = 0; q < v[k]->size(); q++) f[k][q] = (double)(*v[k])[q];
}

// Gravity of a density field: phi by the chosen ordering, g by M2:225-235.
PoissonResult gravity(const cc_mhd2d_params* c, const std::vector<double>& rho, std::vector<double>& gx,
                      std::vector<double>& gy, int mode) {
    PoissonSpec s = m2spec(c);
    PoissonResult r;
    size_t N = (size_t)c->Nx * c->Ny;
    if (!c->gravity_on) { gx.assign(N, 0.0); gy.assign(N, 0.0); return r; }
    std::vector<double> phi;
    if (mode == 2) {
        fft_periodic(s, rho, phi);
    } else if (mode == 3) {
        std::vector<double> rhs = direct_rhs(s, rho);
        direct_solve(s, rhs, phi);
        r.residual = residual_max(s, phi, rhs);
    } else {
        std::vector<double> rhs = poisson_rhs(s, rho);
        r = mode == 0 ? sor_lexicographic(s, rhs, phi) : sor_red_black(s, rhs, phi);
    }
    gravity_from_phi(s, phi, gx, gy);
    return r;
}

M3Par m3par(const cc_mhd3d_params* c) {
    M3Par p;
    p.gamma1 = c->gamma1; p.gamma2 = c->gamma2; p.K1 = c->K1; p.rho_nuc = c->rho_nuc; p.gamma_th = c->gamma_th;
    p.rho_bounce = c->rho_bounce; p.gamma_bounce = c->gamma_bounce; p.Kbounce = c->Kbounce; p.cfl = c->cfl;
    p.x0 = c->x0; p.x1 = c->x1; p.y0 = c->y0; p.y1 = c->y1; p.z0 = c->z0; p.z1 = c->z1;
    p.nx = c->Nx; p.ny = c->Ny; p.nz = c->Nz;
    p.floor_rho = c->floor_rho; p.floor_P = c->floor_P;
    p.px = c->periodic_x != 0; p.py = c->periodic_y != 0; p.pz = c->periodic_z != 0;
    p.eta = c->eta;
    return p;
}

template <class T> void load3(const cc_mhd3d_params* c, const double* const* f, M3State<T>& s) {
    size_t nx = c->Nx, ny = c->Ny, nz = c->Nz, N = nx * ny * nz;
    std::vector<T>* cell[5] = {&s.rho, &s.mx, &s.my, &s.mz, &s.E};
    for (int k = 0; k < 5; k++) cell[k]->assign(f[k], f[k] + N);
    s.bxf.assign(f[5], f[5] + (nx + 1) * ny * nz);
    s.byf.assign(f[6], f[6] + nx * (ny + 1) * nz);
    s.bzf.assign(f[7], f[7] + nx * ny * (nz + 1));
}

template <class T> void store3(const M3State<T>& s, double* const* f) {
    const std::vector<T>* v[8] = {&s.rho, &s.mx, &s.my, &s.mz, &s.E, &s.bxf, &s.byf, &s.bzf};
    for (int k = 0; k < 8; k++)
        for (size_t q = 0; q < v[k]->size(); q++) f[k][q] = (double)(*v[k])[q];
}

template <class T> int main_loop3(const cc_mhd3d_params* c, double* const* f, int nsteps, double* t) {
    M3State<T> s;
    load3(c, f, s);
    M3<T> m(m3par(c));
    double tt = t ? *t : 0.0;
    for (int n = 0; n < nsteps && tt < c->t_end; ++n) {  // M3:1285-1291
        double dt = m.compute_dt(s);
        if (tt + dt > c->t_end) dt = c->t_end - tt;
        m.rk2_step(s, T(dt));
        tt += dt;
    }
    store3(s, f);
    if (t) *t = tt;
    return 0;
}

EHPar ehpar(const cc_euler2d_params* c) {
    EHPar p;
    p.gamma = c->gamma; p.cfl = c->cfl;
    p.x0 = c->x0; p.x1 = c->x1; p.y0 = c->y0; p.y1 = c->y1;
    p.nx = c->Nx; p.ny = c->Ny;
    p.floor_rho = c->floor_rho; p.floor_P = c->floor_P;
    p.px = c->periodic_x != 0; p.py = c->periodic_y != 0;
    p.gravity = c->gravity_on != 0;
    return p;
}

// EH's Poisson: floored density, always periodic (EH:300-323)
PoissonSpec ehspec(const cc_euler2d_params* c) {
    PoissonSpec s;
    s.nx = c->Nx; s.ny = c->Ny; s.px = true; s.py = true;
    s.dx = (c->x1 - c->x0) / c->Nx; s.dy = (c->y1 - c->y0) / c->Ny;
    s.G = c->G; s.omega = c->sor_omega; s.max_iter = c->sor_max_iter; s.tol = c->sor_tol;
    s.floor_density = true; s.floor_rho = c->floor_rho;
    s.Lx = c->x1 - c->x0; s.Ly = c->y1 - c->y0;
    return s;
}

// compute_enclosed_mass_gravity (EH:226-286): cells sorted by distance from
// the domain centre, ties within 1e-12 of a group's first radius grouped,
// enclosed mass summed in sorted order up to the end of each group,
// g = -G M_enc / (r^2 + softening^2) along r-hat.
void enclosed_mass_gravity(const cc_euler2d_params* c, const std::vector<double>& rho, std::vector<double>& gx,
                           std::vector<double>& gy) {
    const int nx = c->Nx, ny = c->Ny;
    gx.assign((size_t)nx * ny, 0.0);
    gy.assign((size_t)nx * ny, 0.0);
    const double dx = (c->x1 - c->x0) / nx, dy = (c->y1 - c->y0) / ny;
    const double cx = 0.5 * (c->x0 + c->x1), cy = 0.5 * (c->y0 + c->y1);
    struct Cell { double r; size_t k; double m, x, y; };
    std::vector<Cell> cells;
    cells.reserve((size_t)nx * ny);
    for (int j = 0; j < ny; ++j) {
        const double y = c->y0 + (j + 0.5) * dy;
        for (int i = 0; i < nx; ++i) {
            const double x = c->x0 + (i + 0.5) * dx;
            const size_t k = (size_t)j * nx + i;
            const double rx = x - cx, ry = y - cy;
            cells.push_back({std::sqrt(rx * rx + ry * ry), k, std::max(rho[k], c->floor_rho) * dx * dy, x, y});
        }
    }
    std::sort(cells.begin(), cells.end(), [](const Cell& a, const Cell& b) { return a.r < b.r; });
    double menc = 0.0;
    size_t s = 0;
    while (s < cells.size()) {
        const double r0 = cells[s].r;
        size_t e = s + 1;
        while (e < cells.size() && cells[e].r <= r0 + 1e-12) ++e;
        for (size_t t = s; t < e; ++t) menc += cells[t].m;
        for (size_t t = s; t < e; ++t) {
            const double rx = cells[t].x - cx, ry = cells[t].y - cy;
            const double r2 = rx * rx + ry * ry + c->softening * c->softening;
            const double r = std::sqrt(r2);
            if (r > 0.0) {
                const double gmag = -c->G * menc / r2;
                gx[cells[t].k] = gmag * (rx / r);
                gy[cells[t].k] = gmag * (ry / r);
            }
        }
        s = e;
    }
}

// Shell-binned enclosed-mass gravity (gravity_accel_from_enclosed_mass,
// gravity_enclosed.h:18-96): r_max over the cell centres (at least 1e-12),
// Nr = max(8, Nr_bins) shells of width r_max / Nr about (xc, yc); the floored
// cell masses deposited into shells in index order, their running sum over
// shells, g = -G M(<shell) r_vec / (r^2 + softening^2)^(3/2).
void shell_mass_gravity(const cc_euler2d_params* c, const std::vector<double>& rho, std::vector<double>& gx,
                        std::vector<double>& gy) {
    const int nx = c->Nx, ny = c->Ny;
    const size_t N = (size_t)nx * ny;
    gx.assign(N, 0.0);
    gy.assign(N, 0.0);
    const double dx = (c->x1 - c->x0) / nx, dy = (c->y1 - c->y0) / ny;
    auto xc_of = [&](int i) { return c->x0 + (i + 0.5) * dx; };
    auto yc_of = [&](int j) { return c->y0 + (j + 0.5) * dy; };
    double rmax = 0.0;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double ddx = xc_of(i) - c->xc, ddy = yc_of(j) - c->yc;
            rmax = std::max(rmax, std::sqrt(ddx * ddx + ddy * ddy));
        }
    rmax = std::max(rmax, 1e-12);
    const int nr = std::max(8, c->Nr_bins);
    const double dr = rmax / (double)nr;
    auto bin = [&](double r) {
        int b = (int)std::floor(r / dr);
        return b < 0 ? 0 : (b >= nr ? nr - 1 : b);
    };
    std::vector<double> shell((size_t)nr, 0.0), menc((size_t)nr, 0.0);
    const double dA = dx * dy;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double ddx = xc_of(i) - c->xc, ddy = yc_of(j) - c->yc;
            shell[(size_t)bin(std::sqrt(ddx * ddx + ddy * ddy))] += std::max(rho[(size_t)j * nx + i], c->floor_rho) * dA;
        }
    double run = 0.0;
    for (int b = 0; b < nr; ++b) menc[(size_t)b] = (run += shell[(size_t)b]);
    const double eps2 = c->softening * c->softening;
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) {
            const double ddx = xc_of(i) - c->xc, ddy = yc_of(j) - c->yc;
            const double r2 = ddx * ddx + ddy * ddy;
            const double denom = std::pow(r2 + eps2, 1.5);
            if (denom <= 0.0) continue;
            const double gcoef = -c->G * menc[(size_t)bin(std::sqrt(r2))] / denom;
            gx[(size_t)j * nx + i] = gcoef * ddx;
            gy[(size_t)j * nx + i] = gcoef * ddy;
        }
}

PoissonResult eh_gravity(const cc_euler2d_params* c, const std::vector<double>& rho, std::vector<double>& gx,
                         std::vector<double>& gy, int mode) {
    PoissonSpec s = ehspec(c);
    PoissonResult r;
    size_t N = (size_t)c->Nx * c->Ny;
    if (!c->gravity_on) { gx.assign(N, 0.0); gy.assign(N, 0.0); return r; }
    if (c->poisson_kind == CC_GRAVITY_ENCLOSED) { enclosed_mass_gravity(c, rho, gx, gy); return r; }
    if (c->poisson_kind == CC_GRAVITY_SHELLS) { shell_mass_gravity(c, rho, gx, gy); return r; }
    std::vector<double> phi;
    if (mode == 2) {
        std::vector<double> fr(rho.begin(), rho.end());
        for (auto& v : fr) v = vmax(v, c->floor_rho);
        fft_periodic(s, fr, phi);
    } else {
        std::vector<double> rhs = poisson_rhs(s, rho);
        r = mode == 0 ? sor_lexicographic(s, rhs, phi) : sor_red_black(s, rhs, phi);
    }
    gravity_from_phi(s, phi, gx, gy);
    return r;
}

template <class T> void loadE(const cc_euler2d_params* c, const double* const* f, EHState<T>& s) {
    size_t N = (size_t)c->Nx * c->Ny;
    s.rho.assign(f[0], f[0] + N); s.mx.assign(f[1], f[1] + N); s.my.assign(f[2], f[2] + N); s.E.assign(f[3], f[3] + N);
}
template <class T> void storeE(const EHState<T>& s, double* const* f) {
    const std::vector<T>* v[4] = {&s.rho, &s.mx, &s.my, &s.E};
    for (int k = 0; k < 4; k++)
        for (size_t q = 0; q < v[k]->size(); q++) f[k][q] = (double)(*v[k])[q];
}

template <class T> std::vector<T> cast(const std::vector<double>& v) { return std::vector<T>(v.begin(), v.end()); }
template <class T> std::vector<double> widen(const std::vector<T>& v) { return std::vector<double>(v.begin(), v.end()); }

template <class T>
void rk2(const cc_mhd2d_params* c, M2State<T>& s, const std::vector<double>& gx, const std::vector<double>& gy,
         double dt, int mode) {
    M2<T> m(m2par(c));
    auto poisson = [&](const std::vector<T>& rho, std::vector<T>& ox, std::vector<T>& oy) {
        std::vector<double> x, y;
        gravity(c, widen(rho), x, y, mode);
        ox = cast<T>(x); oy = cast<T>(y);
    };
    m.rk2_step(s, cast<T>(gx), cast<T>(gy), T(dt), poisson);
}

// Gravity of a dual density field: the value by the chosen solve, the
// tangent by the same (linear) direct solve applied to the density tangent
// (direct mode or gravity off only).
void gravity_dual(const cc_mhd2d_params* c, const std::vector<Dual>& rho, std::vector<Dual>& gx,
                  std::vector<Dual>& gy, int mode) {
    const size_t N = rho.size();
    std::vector<double> rv(N), rd(N), x, y, xd(N, 0.0), yd(N, 0.0);
    for (size_t q = 0; q < N; q++) { rv[q] = rho[q].v; rd[q] = rho[q].d; }
    gravity(c, rv, x, y, mode);
    if (c->gravity_on) {
        PoissonSpec sp = m2spec(c);
        std::vector<double> phi;
        direct_solve(sp, direct_rhs(sp, rd), phi);
        gravity_from_phi(sp, phi, xd, yd);
    }
    gx.resize(N); gy.resize(N);
    for (size_t q = 0; q < N; q++) { gx[q] = Dual(x[q], xd[q]); gy[q] = Dual(y[q], yd[q]); }
}

template <class T> int main_loop(const cc_mhd2d_params* c, double* const* f, int nsteps, double* t, int mode) {
    M2State<T> s;
    load(c, f, s);
    M2<T> m(m2par(c));
    double tt = t ? *t : 0.0;
    for (int n = 0; n < nsteps && tt < c->t_end; ++n) {
        std::vector<double> gx, gy;
        gravity(c, widen(s.rho), gx, gy, mode);
        double dt = m.compute_dt(s);
        if (tt + dt > c->t_end) dt = c->t_end - tt;
        rk2<T>(c, s, gx, gy, dt, mode);
        tt += dt;
    }
    store(s, f);
    if (t) *t = tt;
    return 0;
}
// ---- 2D Navier-Stokes helpers + FFT gravity, HLLC (navier_stokes_2d_hllc_poisson.cpp) ----
NSPar nspar(const cc_ns2d_params* c) {
    NSPar p;
    p.gamma = c->gamma; p.cfl = c->cfl;
    p.x0 = c->x0; p.x1 = c->x1; p.y0 = c->y0; p.y1 = c->y1;
    p.nx = c->Nx; p.ny = c->Ny;
    p.floor_rho = c->floor_rho; p.floor_P = c->floor_P;
    p.viscosity = c->viscosity_on != 0; p.mu = c->mu; p.cfl_visc = c->cfl_visc;
    p.gravity = c->gravity_on != 0; p.G = c->G;
    return p;
}

// the spectral potential (NS:285-328) of a density in T, solved in double
template <class T> typename NS<T>::Potential ns_potential(const cc_ns2d_params* c) {
    return [c](const std::vector<T>& rho, std::vector<T>& phi) {
        PoissonSpec s{};
        s.nx = c->Nx; s.ny = c->Ny; s.px = s.py = true;
        s.dx = (c->x1 - c->x0) / c->Nx; s.dy = (c->y1 - c->y0) / c->Ny;
        s.G = c->G; s.Lx = c->x1 - c->x0; s.Ly = c->y1 - c->y0;
        std::vector<double> r(rho.begin(), rho.end()), ph;
        fft_periodic(s, r, ph);
        phi.assign(ph.begin(), ph.end());
    };
}

template <class T> void loadN(const cc_ns2d_params* c, const double* const* f, NSState<T>& s) {
    const size_t n = (size_t)c->Nx * c->Ny;
    std::vector<T>* d[4] = {&s.d, &s.mx, &s.my, &s.E};
    for (int k = 0; k < 4; k++) d[k]->assign(f[k], f[k] + n);
}
template <class T> void storeN(const NSState<T>& s, double* const* f) {
    const std::vector<T>* d[4] = {&s.d, &s.mx, &s.my, &s.E};
    for (int k = 0; k < 4; k++)
        if (f[k])
            for (size_t q = 0; q < d[k]->size(); q++) f[k][q] = (double)(*d[k])[q];
}

}  // namespace

extern "C" {

int or_mhd2d_gravity(const cc_mhd2d_params* c, const double* rho, double* gx, double* gy, int mode,
                     int* iters, double* residual) {
    std::vector<double> r(rho, rho + (size_t)c->Nx * c->Ny), x, y;
    PoissonResult res = gravity(c, r, x, y, mode);
    std::memcpy(gx, x.data(), x.size() * sizeof(double));
    std::memcpy(gy, y.data(), y.size() * sizeof(double));
    if (iters) *iters = res.iters;
    if (residual) *residual = res.residual;
    return 0;
}

int or_mhd2d_phi(const cc_mhd2d_params* c, const double* rho, double* phi_out, int mode, int* iters,
                 double* residual) {
    PoissonSpec s = m2spec(c);
    std::vector<double> r(rho, rho + (size_t)c->Nx * c->Ny), phi;
    PoissonResult res;
    if (mode == 2) fft_periodic(s, r, phi);
    else if (mode == 3) {
        std::vector<double> rhs = direct_rhs(s, r);
        direct_solve(s, rhs, phi);
        res.residual = residual_max(s, phi, rhs);
    } else {
        std::vector<double> rhs = poisson_rhs(s, r);
        res = mode == 0 ? sor_lexicographic(s, rhs, phi) : sor_red_black(s, rhs, phi);
    }
    std::memcpy(phi_out, phi.data(), phi.size() * sizeof(double));
    if (iters) *iters = res.iters;
    if (residual) *residual = res.residual;
    return 0;
}

double or_mhd2d_compute_dt(const cc_mhd2d_params* c, const double* const* f) {
    M2State<double> s;
    load(c, f, s);
    return M2<double>(m2par(c)).compute_dt(s);
}

int or_mhd2d_advance_stage(const cc_mhd2d_params* c, const double* const* fin, double* const* fout,
                           const double* gx, const double* gy, double dt) {
    M2State<double> s0, s1;
    load(c, fin, s0);
    size_t N = (size_t)c->Nx * c->Ny;
    std::vector<double> x = gx ? std::vector<double>(gx, gx + N) : std::vector<double>(N, 0.0);
    std::vector<double> y = gy ? std::vector<double>(gy, gy + N) : std::vector<double>(N, 0.0);
    M2<double>(m2par(c)).advance_stage(s0, s1, x, y, dt);
    store(s1, fout);
    return 0;
}

int or_mhd2d_rk2_step(const cc_mhd2d_params* c, double* const* f, const double* gx, const double* gy,
                      double dt, int mode) {
    M2State<double> s;
    load(c, f, s);
    size_t N = (size_t)c->Nx * c->Ny;
    std::vector<double> x = gx ? std::vector<double>(gx, gx + N) : std::vector<double>(N, 0.0);
    std::vector<double> y = gy ? std::vector<double>(gy, gy + N) : std::vector<double>(N, 0.0);
    rk2<double>(c, s, x, y, dt, mode);
    store(s, f);
    return 0;
}

// nsteps of the main() loop body (M2:1111-1117) in double (fp32 == 0) or float.
// Tangent-linear model of nsteps of the main-loop body with the dt sequence
// dts (dt held constant): f = values (updated in place, bitwise the double
// run), fd = tangents (updated to J fd).  Gravity: direct solve (mode 3) or off.
int or_mhd2d_tlm(const cc_mhd2d_params* c, double* const* f, double* const* fd, int nsteps, const double* dts) {
    if (c->gravity_on && c->poisson_kind != 2) return -1;
    M2State<Dual> s;
    const size_t N = (size_t)c->Nx * c->Ny, NX = (size_t)(c->Nx + 1) * c->Ny, NY = (size_t)c->Nx * (c->Ny + 1);
    std::vector<Dual>* v[8] = {&s.rho, &s.mx, &s.my, &s.mz, &s.E, &s.Bz, &s.bxf, &s.byf};
    const size_t sz[8] = {N, N, N, N, N, N, NX, NY};
    for (int k = 0; k < 8; k++) {
        v[k]->resize(sz[k]);
        for (size_t q = 0; q < sz[k]; q++) (*v[k])[q] = Dual(f[k][q], fd[k][q]);
    }
    M2<Dual> m(m2par(c));
    auto poisson = [&](const std::vector<Dual>& rho, std::vector<Dual>& ox, std::vector<Dual>& oy) {
        gravity_dual(c, rho, ox, oy, 3);
    };
    for (int n = 0; n < nsteps; ++n) {
        std::vector<Dual> gx, gy;
        gravity_dual(c, s.rho, gx, gy, 3);
        m.rk2_step(s, gx, gy, Dual(dts[n]), poisson);
    }
    for (int k = 0; k < 8; k++)
        for (size_t q = 0; q < sz[k]; q++) { f[k][q] = (*v[k])[q].v; fd[k][q] = (*v[k])[q].d; }
    return 0;
}

int or_mhd2d_main_loop(const cc_mhd2d_params* c, double* const* f, int nsteps, double* t, int mode, int fp32) {
    return fp32 ? main_loop<float>(c, f, nsteps, t, mode) : main_loop<double>(c, f, nsteps, t, mode);
}

double or_mhd2d_divB_max(const cc_mhd2d_params* c, const double* const* f) {
    M2State<double> s;
    load(c, f, s);
    return M2<double>(m2par(c)).max_divB(s);
}

void or_mhd2d_derived(const cc_mhd2d_params* c, const double* const* f, double* const* out) {
    M2State<double> s;
    load(c, f, s);
    M2<double>(m2par(c)).derived(s, out);
}

// ---- 3D MHD (mhd3d_resistive_hlld_ct.cpp) ----
int or_mhd3d_advance_stage(const cc_mhd3d_params* c, const double* const* fin, double* const* fout, double dt) {
    M3State<double> s0, s1;
    load3(c, fin, s0);
    M3<double>(m3par(c)).advance_stage(s0, s1, dt);
    store3(s1, fout);
    return 0;
}

int or_mhd3d_rk2_step(const cc_mhd3d_params* c, double* const* f, double dt) {
    M3State<double> s;
    load3(c, f, s);
    M3<double>(m3par(c)).rk2_step(s, dt);
    store3(s, f);
    return 0;
}

double or_mhd3d_compute_dt(const cc_mhd3d_params* c, const double* const* f) {
    M3State<double> s;
    load3(c, f, s);
    return M3<double>(m3par(c)).compute_dt(s);
}

int or_mhd3d_main_loop(const cc_mhd3d_params* c, double* const* f, int nsteps, double* t, int fp32) {
    return fp32 ? main_loop3<float>(c, f, nsteps, t) : main_loop3<double>(c, f, nsteps, t);
}

void or_mhd3d_derived(const cc_mhd3d_params* c, const double* const* f, double* const* out) {
    M3State<double> s;
    load3(c, f, s);
    M3<double>(m3par(c)).derived(s, out);
}

double or_mhd3d_divB_max(const cc_mhd3d_params* c, const double* const* f) {
    M3State<double> s;
    load3(c, f, s);
    return M3<double>(m3par(c)).max_divB(s);
}

// ---- 2D Euler + gravity, HLLC (euler2d_gravity_hllc.cpp) ----
int or_euler2d_gravity(const cc_euler2d_params* c, const double* rho, double* gx, double* gy, int mode, int* iters,
                       double* residual) {
    std::vector<double> r(rho, rho + (size_t)c->Nx * c->Ny), x, y;
    PoissonResult res = eh_gravity(c, r, x, y, mode);
    std::memcpy(gx, x.data(), x.size() * sizeof(double));
    std::memcpy(gy, y.data(), y.size() * sizeof(double));
    if (iters) *iters = res.iters;
    if (residual) *residual = res.residual;
    return 0;
}

int or_euler2d_rhs(const cc_euler2d_params* c, const double* const* f, double* const* dU, int mode) {
    EHState<double> s;
    loadE(c, f, s);
    std::vector<double> gx, gy;
    eh_gravity(c, s.rho, gx, gy, mode);
    EHState<double> d = EH<double>(ehpar(c)).rhs(s, gx, gy);
    storeE(d, dU);
    return 0;
}

void or_euler2d_derived(const cc_euler2d_params* c, const double* const* f, double* const* out) {
    EHState<double> s;
    loadE(c, f, s);
    EH<double>(ehpar(c)).derived(s, out);
}

double or_euler2d_compute_dt(const cc_euler2d_params* c, const double* const* f) {
    EHState<double> s;
    loadE(c, f, s);
    return EH<double>(ehpar(c)).compute_dt(s);
}

int or_euler2d_rk2_step(const cc_euler2d_params* c, double* const* f, double dt, int mode) {
    EHState<double> s;
    loadE(c, f, s);
    auto grav = [&](const EHState<double>& U, std::vector<double>& gx, std::vector<double>& gy) {
        eh_gravity(c, U.rho, gx, gy, mode);
    };
    EH<double>(ehpar(c)).rk2_step(s, dt, grav);
    storeE(s, f);
    return 0;
}

// main() loop body (EH:697-706) in double (fp32 == 0) or float; returns
// CC_ERR_NONFINITE on a bad dt like the reference's abort (EH:699-702)
int or_euler2d_main_loop(const cc_euler2d_params* c, double* const* f, int nsteps, double* t, int mode, int fp32) {
    auto run = [&](auto tag) -> int {
        using T = decltype(tag);
        EHState<T> s;
        loadE(c, f, s);
        EH<T> m(ehpar(c));
        auto grav = [&](const EHState<T>& U, std::vector<T>& gx, std::vector<T>& gy) {
            std::vector<double> x, y;
            eh_gravity(c, widen(U.rho), x, y, mode);
            gx = cast<T>(x); gy = cast<T>(y);
        };
        double tt = t ? *t : 0.0;
        int rc = 0;
        for (int n = 0; n < nsteps && tt < c->t_end - 1e-14; ++n) {
            double dt = m.compute_dt(s);
            if (!std::isfinite(dt) || dt <= 0.0) { rc = CC_ERR_NONFINITE; break; }
            if (tt + dt > c->t_end) dt = c->t_end - tt;
            m.rk2_step(s, T(dt), grav);
            tt += dt;
        }
        storeE(s, f);
        if (t) *t = tt;
        return rc;
    };
    return fp32 ? run(0.0f) : run(0.0);
}

// ---- 2D Navier-Stokes + FFT gravity, HLLC (navier_stokes_2d_hllc_poisson.cpp) ----
int or_ns2d_ic(const cc_ns2d_params* c, double* const* f) {
    NSState<double> s;
    ns_ic_collapse(nspar(c), c->seed, s);
    storeN(s, f);
    return 0;
}

// phi of the state's cons_to_prim density and g = -grad phi (NS:372-383)
int or_ns2d_gravity(const cc_ns2d_params* c, const double* const* f, double* phi, double* gx, double* gy) {
    NSState<double> s;
    loadN(c, f, s);
    NS<double> m(nspar(c));
    std::vector<double> rho(s.d.size()), ph, x, y;
    for (size_t q = 0; q < rho.size(); q++) rho[q] = m.prim(s.d[q], s.mx[q], s.my[q], s.E[q]).d;
    ns_potential<double>(c)(rho, ph);
    m.gravity_accel(ph, x, y);
    if (phi) std::memcpy(phi, ph.data(), ph.size() * sizeof(double));
    if (gx) std::memcpy(gx, x.data(), x.size() * sizeof(double));
    if (gy) std::memcpy(gy, y.data(), y.size() * sizeof(double));
    return 0;
}

int or_ns2d_rhs(const cc_ns2d_params* c, const double* const* f, double* const* dU) {
    NSState<double> s;
    loadN(c, f, s);
    storeN(NS<double>(nspar(c)).rhs(s, ns_potential<double>(c)), dU);
    return 0;
}

double or_ns2d_compute_dt(const cc_ns2d_params* c, const double* const* f) {
    NSState<double> s;
    loadN(c, f, s);
    return NS<double>(nspar(c)).compute_dt(s);
}

int or_ns2d_rk2_step(const cc_ns2d_params* c, double* const* f, double dt) {
    NSState<double> s;
    loadN(c, f, s);
    NS<double>(nspar(c)).heun(s, dt, ns_potential<double>(c));
    storeN(s, f);
    return 0;
}

void or_ns2d_derived(const cc_ns2d_params* c, const double* const* f, double* const* out) {
    NSState<double> s;
    loadN(c, f, s);
    NS<double>(nspar(c)).derived(s, ns_potential<double>(c), out);
}

// main() loop body (NS:758-791) in double (fp32 == 0) or float
int or_ns2d_main_loop(const cc_ns2d_params* c, double* const* f, int nsteps, double* t, int fp32) {
    auto run = [&](auto tag) -> int {
        using T = decltype(tag);
        NSState<T> s;
        loadN(c, f, s);
        NS<T> m(nspar(c));
        const auto pot = ns_potential<T>(c);
        double tt = t ? *t : 0.0;
        for (int n = 0; n < nsteps && tt < c->t_end - 1e-14; ++n) {
            double dt = m.compute_dt(s);
            if (tt + dt > c->t_end) dt = c->t_end - tt;
            m.heun(s, T(dt), pot);
            tt += dt;
        }
        storeN(s, f);
        if (t) *t = tt;
        return 0;
    };
    return fp32 ? run(0.0f) : run(0.0);
}

// Gravity of a density field with every Poisson knob explicit (used to pin the
// restated SOR against both reference variants: M2's fixed sweeps and EH's
// floored-density, residual-tolerance solve).
int or_poisson_generic(int nx, int ny, int px, int py, double dx, double dy, double G, double omega, int max_iter,
                       double tol, int floor_density, double floor_rho, int mode, const double* rho, double* gx,
                       double* gy, int* iters, double* residual) {
    PoissonSpec s;
    s.nx = nx; s.ny = ny; s.px = px != 0; s.py = py != 0; s.dx = dx; s.dy = dy; s.G = G; s.omega = omega;
    s.max_iter = max_iter; s.tol = tol; s.floor_density = floor_density != 0; s.floor_rho = floor_rho;
    s.Lx = nx * dx; s.Ly = ny * dy;
    std::vector<double> r(rho, rho + (size_t)nx * ny), phi, x, y;
    PoissonResult res;
    if (mode == 2) fft_periodic(s, r, phi);
    else {
        std::vector<double> rhs = poisson_rhs(s, r);
        res = mode == 0 ? sor_lexicographic(s, rhs, phi) : sor_red_black(s, rhs, phi);
    }
    gravity_from_phi(s, phi, x, y);
    std::memcpy(gx, x.data(), x.size() * sizeof(double));
    std::memcpy(gy, y.data(), y.size() * sizeof(double));
    if (iters) *iters = res.iters;
    if (residual) *residual = res.residual;
    return 0;
}

// Standalone FFT pieces for the tests.
int or_fft1d(int n, double* reim, int inverse) {
    std::vector<std::complex<double>> a(n);
    for (int i = 0; i < n; i++) a[i] = {reim[2 * i], reim[2 * i + 1]};
    fft_1d(a, inverse != 0);
    for (int i = 0; i < n; i++) { reim[2 * i] = a[i].real(); reim[2 * i + 1] = a[i].imag(); }
    return 0;
}

}  // extern "C"
