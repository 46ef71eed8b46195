// ORACLE / TEST INFRASTRUCTURE ONLY.  Nothing in core_collapse_b200 links or
// calls this file.  It compiles the reference solver
// mhd2d_resistive_hlld_ct_gravity.cpp *in place* (from the reference tree, via
// -I, never copied) inside a private namespace, and exports its static
// functions through a C ABI so tests can run the reference itself:
//   rk2_step                         M2:838-869
//   advance_stage                    M2:690-834
//   compute_dt                       M2:579-598
//   compute_poisson_gravity_periodic M2:178-237
//   the main() loop body             M2:1111-1117
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <iomanip>
#include <iostream>
#include <random>
#include <string>
#include <vector>
#include "hdf5.h"
#include "../include/cc_step.h"

#define main ref_mhd2d_main
namespace refm2 {
#include "mhd2d_resistive_hlld_ct_gravity.cpp"
}
#undef main

namespace {
using namespace refm2;

Params to_params(const cc_mhd2d_params* c) {
    Params p;
    p.gamma = c->gamma; p.cfl = c->cfl;
    p.x0 = c->x0; p.x1 = c->x1; p.y0 = c->y0; p.y1 = c->y1;
    p.Nx = c->Nx; p.Ny = c->Ny;
    p.t_end = c->t_end; p.dt_store = c->dt_store;
    p.floor_rho = c->floor_rho; p.floor_P = c->floor_P;
    p.periodic_x = c->periodic_x != 0; p.periodic_y = c->periodic_y != 0;
    p.eta = c->eta;
    p.gravity_on = c->gravity_on != 0;
    p.G = c->G; p.softening = c->softening;
    p.sor_iters = c->sor_iters; p.sor_omega = c->sor_omega;
    return p;
}

void load(const Params& p, const double* const* f, Ucc& U, Bfaces& B) {
    size_t N = (size_t)p.Nx * p.Ny, NX = (size_t)(p.Nx + 1) * p.Ny, NY = (size_t)p.Nx * (p.Ny + 1);
    U.rho.assign(f[0], f[0] + N); U.mx.assign(f[1], f[1] + N); U.my.assign(f[2], f[2] + N);
    U.mz.assign(f[3], f[3] + N); U.E.assign(f[4], f[4] + N); U.Bz.assign(f[5], f[5] + N);
    B.Bx_f.assign(f[6], f[6] + NX); B.By_f.assign(f[7], f[7] + NY);
}

void store(const Ucc& U, const Bfaces& B, double* const* f) {
    std::copy(U.rho.begin(), U.rho.end(), f[0]); std::copy(U.mx.begin(), U.mx.end(), f[1]);
    std::copy(U.my.begin(), U.my.end(), f[2]); std::copy(U.mz.begin(), U.mz.end(), f[3]);
    std::copy(U.E.begin(), U.E.end(), f[4]); std::copy(U.Bz.begin(), U.Bz.end(), f[5]);
    std::copy(B.Bx_f.begin(), B.Bx_f.end(), f[6]); std::copy(B.By_f.begin(), B.By_f.end(), f[7]);
}

GravField grav(const Params& p, const double* gx, const double* gy) {
    GravField g;
    size_t N = (size_t)p.Nx * p.Ny;
    if (gx) g.gx.assign(gx, gx + N); else g.gx.assign(N, 0.0);
    if (gy) g.gy.assign(gy, gy + N); else g.gy.assign(N, 0.0);
    return g;
}
}  // namespace

extern "C" {

int ref_mhd2d_rk2_step(const cc_mhd2d_params* c, double* const* f,
                       const double* gx, const double* gy, double dt) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
    GravField g = grav(p, gx, gy);
    rk2_step(p, U, B, g, dx, dy, dt);
    store(U, B, f);
    return 0;
}

int ref_mhd2d_advance_stage(const cc_mhd2d_params* c, double* const* fin, double* const* fout,
                            const double* gx, const double* gy, double dt) {
    Params p = to_params(c);
    Ucc U0, U1; Bfaces B0, B1; load(p, fin, U0, B0);
    double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
    GravField g = grav(p, gx, gy);
    advance_stage(p, U0, B0, U1, B1, g, dx, dy, dt);
    store(U1, B1, fout);
    return 0;
}

double ref_mhd2d_compute_dt(const cc_mhd2d_params* c, double* const* f) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
    return compute_dt(p, U, B, dx, dy);
}

int ref_mhd2d_poisson(const cc_mhd2d_params* c, const double* rho, double* gx, double* gy) {
    Params p = to_params(c);
    std::vector<double> r(rho, rho + (size_t)p.Nx * p.Ny);
    double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
    GravField g = compute_poisson_gravity_periodic(p, r, dx, dy);
    std::copy(g.gx.begin(), g.gx.end(), gx);
    std::copy(g.gy.begin(), g.gy.end(), gy);
    return 0;
}

// nsteps iterations of the main() loop body (M2:1111-1117) without snapshots.
int ref_mhd2d_main_loop(const cc_mhd2d_params* c, double* const* f, int nsteps, double* t) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
    double tt = t ? *t : 0.0;
    for (int n = 0; n < nsteps && tt < p.t_end; ++n) {
        GravField g = compute_poisson_gravity_periodic(p, U.rho, dx, dy);
        double dt = compute_dt(p, U, B, dx, dy);
        if (tt + dt > p.t_end) dt = p.t_end - tt;
        rk2_step(p, U, B, g, dx, dy, dt);
        tt += dt;
    }
    store(U, B, f);
    if (t) *t = tt;
    return 0;
}

double ref_mhd2d_divB_max(const cc_mhd2d_params* c, double* const* f) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx = (p.x1 - p.x0) / p.Nx, dy = (p.y1 - p.y0) / p.Ny;
    double m = 0.0;
    for (int j = 0; j < p.Ny; j++)
        for (int i = 0; i < p.Nx; i++) m = std::max(m, std::abs(divB_cc(p, B, i, j, dx, dy)));
    return m;
}

// The reference's own main() (its defaults, initial condition, time loop and
// snapshot store), run once; its HDF5 datasets are recorded in memory by the
// recording hdf5.h of this directory (read back through cc_h5rec_*).
int ref_mhd2d_run_main() {
    cc_h5rec_clear();
    return refm2::ref_mhd2d_main();
}

}  // extern "C"
