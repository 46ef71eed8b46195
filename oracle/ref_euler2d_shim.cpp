// ORACLE / TEST INFRASTRUCTURE ONLY.  Compiles the reference solver
// euler2d_gravity_hllc.cpp in place (via -I, never copied) inside a private
// namespace and exports, through a C ABI:
//   rk2_step                          EH:529-550
//   rhs                               EH:406-527
//   compute_dt                        EH:390-404
//   compute_poisson_gravity_periodic  EH:288-386 (hard-coded omega 1.7, tol 1e-10, 50000 sweeps)
//   compute_enclosed_mass_gravity     EH:226-286 (the rhs's commented-out alternative, EH:411)
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

#define main ref_euler2d_main
namespace refeh {
#include "euler2d_gravity_hllc.cpp"
}
#undef main

namespace {
using namespace refeh;

Params to_params(const cc_euler2d_params* c) {
    Params p;
    p.gamma = c->gamma; p.cfl = c->cfl;
    p.x0 = c->x0; p.x1 = c->x1; p.y0 = c->y0; p.y1 = c->y1;
    p.Nx = c->Nx; p.Ny = c->Ny;
    p.t_end = c->t_end; p.dt_store = c->dt_store;
    p.floor_rho = c->floor_rho; p.floor_P = c->floor_P;
    p.periodic_x = c->periodic_x != 0; p.periodic_y = c->periodic_y != 0;
    p.gravity_on = c->gravity_on != 0;
    p.G = c->G; p.softening = c->softening;
    return p;
}

void load(const Params& p, const double* const* f, State& U) {
    size_t N = (size_t)p.Nx * p.Ny;
    U.rho.assign(f[0], f[0] + N); U.mx.assign(f[1], f[1] + N);
    U.my.assign(f[2], f[2] + N); U.E.assign(f[3], f[3] + N);
}

void store(const State& U, double* const* f) {
    std::copy(U.rho.begin(), U.rho.end(), f[0]); std::copy(U.mx.begin(), U.mx.end(), f[1]);
    std::copy(U.my.begin(), U.my.end(), f[2]); std::copy(U.E.begin(), U.E.end(), f[3]);
}
}  // namespace

extern "C" {

int ref_euler2d_rk2_step(const cc_euler2d_params* c, double* const* f, double dt) {
    Params p = to_params(c);
    State U; load(p, f, U);
    rk2_step(p, U, dt);
    store(U, f);
    return 0;
}

int ref_euler2d_rhs(const cc_euler2d_params* c, const double* const* f, double* const* dU) {
    Params p = to_params(c);
    State U; load(p, f, U);
    State d = rhs(p, U);
    store(d, dU);
    return 0;
}

double ref_euler2d_compute_dt(const cc_euler2d_params* c, const double* const* f) {
    Params p = to_params(c);
    State U; load(p, f, U);
    return compute_dt(p, U);
}

int ref_euler2d_poisson(const cc_euler2d_params* c, const double* const* f, double* gx, double* gy) {
    Params p = to_params(c);
    State U; load(p, f, U);
    GravField g = compute_poisson_gravity_periodic(p, U);
    std::copy(g.gx.begin(), g.gx.end(), gx);
    std::copy(g.gy.begin(), g.gy.end(), gy);
    return 0;
}

int ref_euler2d_enclosed_gravity(const cc_euler2d_params* c, const double* const* f, double* gx, double* gy) {
    Params p = to_params(c);
    State U; load(p, f, U);
    GravField g = compute_enclosed_mass_gravity(p, U);
    std::copy(g.gx.begin(), g.gx.end(), gx);
    std::copy(g.gy.begin(), g.gy.end(), gy);
    return 0;
}

int ref_euler2d_init_random_blob(const cc_euler2d_params* c, double* const* f) {
    Params p = to_params(c);
    State U = init_random_blob(p);
    store(U, f);
    return 0;
}

int ref_euler2d_main_loop(const cc_euler2d_params* c, double* const* f, int nsteps, double* t) {
    Params p = to_params(c);
    State U; load(p, f, U);
    double tt = t ? *t : 0.0;
    for (int n = 0; n < nsteps && tt < p.t_end - 1e-14; ++n) {
        double dt = compute_dt(p, U);
        if (!std::isfinite(dt) || dt <= 0.0) return -4;
        if (tt + dt > p.t_end) dt = p.t_end - tt;
        rk2_step(p, U, dt);
        tt += dt;
    }
    store(U, f);
    if (t) *t = tt;
    return 0;
}

}  // extern "C"
