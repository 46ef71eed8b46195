// Host set-up of the 3D constant block from the C parameters (shared by the
// solver handle and the host initial condition).
#pragma once
#include <cmath>

#include "../../include/cc_step.h"
#include "mhd3d_physics.cuh"

namespace ccb {

template <class T> M3Const<T> m3_make_const(const cc_mhd3d_params& p) {
    M3Const<T> c{};
    const int nx = p.Nx, ny = p.Ny, nz = p.Nz;
    const double dx = (p.x1 - p.x0) / nx, dy = (p.y1 - p.y0) / ny, dz = (p.z1 - p.z0) / nz;
    // EOS constants; the powers at rho_nuc / rho_bounce use the host's std::pow,
    // as the reference evaluates them on every call (M3:120, 129-130, 135-137)
    const double K2 = p.K1 * std::pow(p.rho_nuc, p.gamma1 - p.gamma2);
    c.g1 = (T)p.gamma1; c.g2 = (T)p.gamma2; c.K1 = (T)p.K1; c.K2 = (T)K2; c.rn = (T)p.rho_nuc;
    c.gth = (T)p.gamma_th; c.rb = (T)p.rho_bounce; c.gb = (T)p.gamma_bounce; c.Kb = (T)p.Kbounce;
    c.g1m1 = (T)(p.gamma1 - 1.0); c.g2m1 = (T)(p.gamma2 - 1.0); c.gbm1 = (T)(p.gamma_bounce - 1.0);
    c.gthm1 = (T)(p.gamma_th - 1.0);
    c.e1n = (T)(p.K1 * std::pow(p.rho_nuc, p.gamma1 - 1.0) / (p.gamma1 - 1.0));
    c.e2n = (T)(K2 * std::pow(p.rho_nuc, p.gamma2 - 1.0) / (p.gamma2 - 1.0));
    c.pbb = (T)std::pow(p.rho_bounce, p.gamma_bounce);
    c.ebb = (T)std::pow(p.rho_bounce, p.gamma_bounce - 1.0);
    c.cold_off = (p.K1 == 0.0 && p.Kbounce == 0.0) ? 1 : 0;
    c.floor_rho = (T)p.floor_rho; c.floor_P = (T)p.floor_P; c.eta = (T)p.eta;
    c.dx = (T)dx; c.dy = (T)dy; c.dz = (T)dz;
    c.inv_dx = (T)(1.0 / dx); c.inv_dy = (T)(1.0 / dy); c.inv_dz = (T)(1.0 / dz);
    c.two_dx = (T)(2.0 * dx); c.two_dy = (T)(2.0 * dy); c.two_dz = (T)(2.0 * dz);
    c.nx = nx; c.ny = ny; c.nz = nz;
    c.P = ((nx + 1 + 31) / 32) * 32;
    c.PS = (long long)c.P * (ny + 1);
    c.ax = AxisMap{nx, p.periodic_x ? 1 : 0};
    c.ay = AxisMap{ny, p.periodic_y ? 1 : 0};
    c.az = AxisMap{nz, p.periodic_z ? 1 : 0};
    c.resistive = (p.eta > 0.0) ? 1 : 0;
    return c;
}

}  // namespace ccb
