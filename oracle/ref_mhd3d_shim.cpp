// ORACLE / TEST INFRASTRUCTURE ONLY.  Compiles the reference solver
// mhd3d_resistive_hlld_ct.cpp in place (via -I, never copied) inside a private
// namespace and exports, through a C ABI:
//   rk2_step       M3:1034-1066
//   advance_stage  M3:694-1030
//   compute_dt     M3:626-648
//   divB_cc        M3:1070-1078
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

#define main ref_mhd3d_main
namespace refm3 {
#include "mhd3d_resistive_hlld_ct.cpp"
}
#undef main

namespace {
using namespace refm3;

Params to_params(const cc_mhd3d_params* c) {
    Params p;
    p.gamma1 = c->gamma1; p.gamma2 = c->gamma2; p.K1 = c->K1; p.rho_nuc = c->rho_nuc;
    p.gamma_th = c->gamma_th; p.rho_bounce = c->rho_bounce; p.gamma_bounce = c->gamma_bounce;
    p.Kbounce = c->Kbounce; p.gamma_init = c->gamma_init; p.cfl = c->cfl;
    p.x0 = c->x0; p.x1 = c->x1; p.y0 = c->y0; p.y1 = c->y1; p.z0 = c->z0; p.z1 = c->z1;
    p.Nx = c->Nx; p.Ny = c->Ny; p.Nz = c->Nz;
    p.t_end = c->t_end; p.dt_store = c->dt_store;
    p.floor_rho = c->floor_rho; p.floor_P = c->floor_P;
    p.periodic_x = c->periodic_x != 0; p.periodic_y = c->periodic_y != 0; p.periodic_z = c->periodic_z != 0;
    p.eta = c->eta;
    return p;
}

void load(const Params& p, const double* const* f, Ucc& U, Bfaces& B) {
    size_t nx = p.Nx, ny = p.Ny, nz = p.Nz;
    size_t N = nx * ny * nz;
    U.rho.assign(f[0], f[0] + N); U.mx.assign(f[1], f[1] + N); U.my.assign(f[2], f[2] + N);
    U.mz.assign(f[3], f[3] + N); U.E.assign(f[4], f[4] + N);
    B.Bx_f.assign(f[5], f[5] + (nx + 1) * ny * nz);
    B.By_f.assign(f[6], f[6] + nx * (ny + 1) * nz);
    B.Bz_f.assign(f[7], f[7] + nx * ny * (nz + 1));
}

void store(const Ucc& U, const Bfaces& B, double* const* f) {
    std::copy(U.rho.begin(), U.rho.end(), f[0]); std::copy(U.mx.begin(), U.mx.end(), f[1]);
    std::copy(U.my.begin(), U.my.end(), f[2]); std::copy(U.mz.begin(), U.mz.end(), f[3]);
    std::copy(U.E.begin(), U.E.end(), f[4]);
    std::copy(B.Bx_f.begin(), B.Bx_f.end(), f[5]); std::copy(B.By_f.begin(), B.By_f.end(), f[6]);
    std::copy(B.Bz_f.begin(), B.Bz_f.end(), f[7]);
}

void spacing(const Params& p, double& dx, double& dy, double& dz) {
    dx = (p.x1 - p.x0) / p.Nx; dy = (p.y1 - p.y0) / p.Ny; dz = (p.z1 - p.z0) / p.Nz;
}
}  // namespace

extern "C" {

int ref_mhd3d_rk2_step(const cc_mhd3d_params* c, double* const* f, double dt) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx, dy, dz; spacing(p, dx, dy, dz);
    rk2_step(p, U, B, dx, dy, dz, dt);
    store(U, B, f);
    return 0;
}

int ref_mhd3d_advance_stage(const cc_mhd3d_params* c, double* const* fin, double* const* fout, double dt) {
    Params p = to_params(c);
    Ucc U0, U1; Bfaces B0, B1; load(p, fin, U0, B0);
    double dx, dy, dz; spacing(p, dx, dy, dz);
    advance_stage(p, U0, B0, U1, B1, dx, dy, dz, dt);
    store(U1, B1, fout);
    return 0;
}

double ref_mhd3d_compute_dt(const cc_mhd3d_params* c, double* const* f) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx, dy, dz; spacing(p, dx, dy, dz);
    return compute_dt(p, U, B, dx, dy, dz);
}

int ref_mhd3d_main_loop(const cc_mhd3d_params* c, double* const* f, int nsteps, double* t) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx, dy, dz; spacing(p, dx, dy, dz);
    double tt = t ? *t : 0.0;
    for (int n = 0; n < nsteps && tt < p.t_end; ++n) {
        double dt = compute_dt(p, U, B, dx, dy, dz);
        if (tt + dt > p.t_end) dt = p.t_end - tt;
        rk2_step(p, U, B, dx, dy, dz, dt);
        tt += dt;
    }
    store(U, B, f);
    if (t) *t = tt;
    return 0;
}

double ref_mhd3d_divB_max(const cc_mhd3d_params* c, double* const* f) {
    Params p = to_params(c);
    Ucc U; Bfaces B; load(p, f, U, B);
    double dx, dy, dz; spacing(p, dx, dy, dz);
    double m = 0.0;
    for (int k = 0; k < p.Nz; k++)
        for (int j = 0; j < p.Ny; j++)
            for (int i = 0; i < p.Nx; i++) m = std::max(m, std::abs(divB_cc(p, B, i, j, k, dx, dy, dz)));
    return m;
}

// The reference's own main() (its defaults, initial condition, time loop and
// snapshot store), run once; its HDF5 datasets are recorded in memory by the
// recording hdf5.h of this directory (read back through cc_h5rec_*).
int ref_mhd3d_run_main() {
    cc_h5rec_clear();
    return refm3::ref_mhd3d_main();
}

}  // extern "C"
