// Host initial condition of the 3D reference driver (cc_ic_mhd3d_reference,
// mhd3d_resistive_hlld_ct.cpp:1159-1272).  A .cu unit so that the cells go
// through the same hybrid-EOS functions as the solver (mhd3d_physics.cuh, host
// and device); the host compiler evaluates them in the reference's order.
#include <algorithm>
#include <cmath>
#include <vector>

#include "../../include/cc_ic.h"
#include "mhd3d_const.h"

using namespace ccb;

namespace {

int wrap_or_clamp(int i, int n, int periodic) {   // imod(i, n) or clamp(i, 0, n - 1)
    if (periodic) return ((i % n) + n) % n;
    return std::min(std::max(i, 0), n - 1);
}

}  // namespace

extern "C" {

void cc_mhd3d_ic_knobs_default(cc_mhd3d_ic_knobs* k) {
    if (!k) return;
    k->rho_bg = 1.0; k->rho_core = 20.0; k->r_core = 0.12; k->r_edge = 0.02;
    k->P0 = 0.15; k->vin = 1.25; k->rot_omega = 1.0;
    k->B0x = 0.15; k->B0z = 0.05; k->Bshear = 0.05;
}

int cc_ic_mhd3d_reference(const cc_mhd3d_params* pp, const cc_mhd3d_ic_knobs* kk, double* const* f) {
    if (!pp || !f) return -1;
    for (int m = 0; m < 8; m++)
        if (!f[m]) return -1;
    const cc_mhd3d_params& p = *pp;
    cc_mhd3d_ic_knobs k;
    if (kk) k = *kk;
    else cc_mhd3d_ic_knobs_default(&k);
    const int Nx = p.Nx, Ny = p.Ny, Nz = p.Nz;
    if (Nx < 1 || Ny < 1 || Nz < 1) return -1;
    const double dx = (p.x1 - p.x0) / Nx, dy = (p.y1 - p.y0) / Ny, dz = (p.z1 - p.z0) / Nz;
    const double cx = 0.5 * (p.x0 + p.x1), cy = 0.5 * (p.y0 + p.y1), cz = 0.5 * (p.z0 + p.z1);
    // corner vector potential with the reference's corner wrap (mod N+1) or clamp (M3:1163-1195)
    std::vector<double> Az((size_t)(Nx + 1) * (Ny + 1) * (Nz + 1), 0.0);
    auto az_idx = [&](int ic, int jc, int kc) -> size_t {
        ic = wrap_or_clamp(ic, Nx + 1, p.periodic_x);
        jc = wrap_or_clamp(jc, Ny + 1, p.periodic_y);
        kc = wrap_or_clamp(kc, Nz + 1, p.periodic_z);
        return ((size_t)kc * (Ny + 1) + jc) * (Nx + 1) + ic;
    };
    auto core = [&](double X, double Y, double Z, double& rx, double& ry, double& rz, double& r) {
        rx = X - cx; ry = Y - cy; rz = Z - cz;
        r = std::sqrt(rx * rx + ry * ry + rz * rz) + 1e-14;
        const double s = (r - k.r_core) / std::max(k.r_edge, 1e-12);
        return 0.5 * (1.0 - std::tanh(s));
    };
    for (int kc = 0; kc <= Nz; ++kc)
        for (int jc = 0; jc <= Ny; ++jc)
            for (int ic = 0; ic <= Nx; ++ic) {
                const double X = p.x0 + ic * dx, Y = p.y0 + jc * dy, Z = p.z0 + kc * dz;
                double rx, ry, rz, r;
                const double cs = core(X, Y, Z, rx, ry, rz, r);
                Az[az_idx(ic, jc, kc)] = k.Bshear * cs * std::sin(2.0 * M_PI * X) * std::sin(2.0 * M_PI * Y);
            }
    double* bx = f[5];
    double* by = f[6];
    double* bz = f[7];
    for (int kk2 = 0; kk2 < Nz; kk2++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i <= Nx; i++)
                bx[((size_t)kk2 * Ny + j) * (Nx + 1) + i] = (Az[az_idx(i, j + 1, kk2)] - Az[az_idx(i, j, kk2)]) / dy + k.B0x;
    for (int kk2 = 0; kk2 < Nz; kk2++)
        for (int j = 0; j <= Ny; j++)
            for (int i = 0; i < Nx; i++)
                by[((size_t)kk2 * (Ny + 1) + j) * Nx + i] = -(Az[az_idx(i + 1, j, kk2)] - Az[az_idx(i, j, kk2)]) / dx;
    for (size_t q = 0; q < (size_t)Nx * Ny * (Nz + 1); q++) bz[q] = k.B0z;
    // cells (M3:1228-1268)
    const M3Const<double> c = m3_make_const<double>(p);
    for (int kk2 = 0; kk2 < Nz; kk2++)
        for (int j = 0; j < Ny; j++)
            for (int i = 0; i < Nx; i++) {
                const double X = p.x0 + (i + 0.5) * dx, Y = p.y0 + (j + 0.5) * dy, Z = p.z0 + (kk2 + 0.5) * dz;
                double rx, ry, rz, r;
                const double cs = core(X, Y, Z, rx, ry, rz, r);
                const double rho = k.rho_bg + (k.rho_core - k.rho_bg) * cs;
                const double P = k.P0 * std::pow(rho / k.rho_bg, p.gamma_init);
                double u = 0.0, v = 0.0, w = 0.0;
                const double vin = k.vin * cs;
                u -= vin * rx / r;
                v -= vin * ry / r;
                w -= vin * rz / r;
                if (k.rot_omega != 0.0) {
                    u += -k.rot_omega * (Y - cy);
                    v += k.rot_omega * (X - cx);
                }
                // cell-centred B: the two faces of the cell (an interior cell's faces never wrap)
                const double Bx = 0.5 * (bx[((size_t)kk2 * Ny + j) * (Nx + 1) + i] + bx[((size_t)kk2 * Ny + j) * (Nx + 1) + i + 1]);
                const double By = 0.5 * (by[((size_t)kk2 * (Ny + 1) + j) * Nx + i] + by[((size_t)kk2 * (Ny + 1) + j + 1) * Nx + i]);
                const double Bz = 0.5 * (bz[((size_t)kk2 * Ny + j) * Nx + i] + bz[((size_t)(kk2 + 1) * Ny + j) * Nx + i]);
                Prim<double> W;
                W.r = rho; W.u = u; W.v = v; W.w = w; W.P = P; W.bx = Bx; W.by = By; W.bz = Bz;
                // prim_to_cons (M3:199-204) and enforce_floors (M3:165-183)
                const size_t q = ((size_t)kk2 * Ny + j) * Nx + i;
                double rr = std::max(W.r, p.floor_rho);
                double E = energy(c, W);
                floors(c, rr, rr * u, rr * v, rr * w, E, Bx, By, Bz);
                f[0][q] = rr; f[1][q] = rr * u; f[2][q] = rr * v; f[3][q] = rr * w; f[4][q] = E;
            }
    return 0;
}

}  // extern "C"
