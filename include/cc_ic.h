/*
 * cc_ic.h -- host-side initial conditions of libcc_b200 (no GPU needed).
 *
 * Each function fills FP64 arrays in the reference layouts
 *   f = {rho, mx, my, mz, E, Bz, Bx_f, By_f}
 * (sizes Nx*Ny for the six cell fields, (Nx+1)*Ny for Bx_f, Nx*(Ny+1) for By_f)
 * and returns 0, or -1 on a bad argument.  Cells are set through the
 * reference's prim_to_cons + enforce_floors
 * (mhd2d_resistive_hlld_ct_gravity.cpp:137-146, 114-124).
 */
#ifndef CC_IC_H
#define CC_IC_H

#include <stdint.h>

#include "cc_step.h"

#ifdef __cplusplus
extern "C" {
#endif

/* IC knobs of the reference main() (mhd2d_resistive_hlld_ct_gravity.cpp:74-85, 1011) */
typedef struct cc_mhd2d_ic_knobs {
    double rho_bg, rho_core, r_core, r_edge, P0, vin, rot_omega;
    double B0x, Bshear;
    double gamma_eff;   /* 1.05, the pressure exponent of M2:1011 */
} cc_mhd2d_ic_knobs;

void cc_mhd2d_ic_knobs_default(cc_mhd2d_ic_knobs* k);

/* The reference main()'s core-collapse IC (M2:957-1048): corner vector
 * potential Az -> divergence-free faces, tanh core, infall + rotation. */
int cc_ic_mhd2d_reference(const cc_mhd2d_params* p, const cc_mhd2d_ic_knobs* k, double* const* f);

/* Gaussian collapse core with multiplicative noise:
 *   rho = (1 + core_amp exp(-r^2/(2 core_width^2))) (1 + noise U(-1,1)),
 * one std::mt19937(seed) + uniform_real_distribution<double>(-1,1) draw per
 * cell, j outer, i inner; v = 0; P = p0 rho^p_exponent; Bx_f = Bx0, By_f = 0, Bz = 0. */
int cc_ic_mhd2d_collapse(const cc_mhd2d_params* p, double core_amp, double core_width, double noise, uint32_t seed,
                         double Bx0, double p0, double p_exponent, double* const* f);

/* Orszag-Tang fields plus an additive Gaussian density core:
 *   rho = 25/(36 pi) + core_amp exp(-r^2/(2 core_width^2)), P = 5/(12 pi),
 *   v = (-sin 2 pi y, sin 2 pi x), B from Az = B0 (cos(2 pi y)/(2 pi) + cos(4 pi x)/(4 pi)),
 *   B0 = 1/sqrt(4 pi) on corners (div B = 0 to roundoff). */
int cc_ic_mhd2d_orszag_tang(const cc_mhd2d_params* p, double core_amp, double core_width, double* const* f);

/* IC knobs of the 3D reference main() (mhd3d_resistive_hlld_ct.cpp:77-88) */
typedef struct cc_mhd3d_ic_knobs {
    double rho_bg, rho_core, r_core, r_edge, P0, vin, rot_omega;
    double B0x, B0z, Bshear;
} cc_mhd3d_ic_knobs;

void cc_mhd3d_ic_knobs_default(cc_mhd3d_ic_knobs* k);

/* The 3D reference main()'s core-collapse IC (M3:1159-1272): corner vector
 * potential Az = Bshear core(r) sin(2 pi X) sin(2 pi Y) -> Bx_f = dAz/dy + B0x,
 * By_f = -dAz/dx, Bz_f = B0z; tanh core, P = P0 (rho/rho_bg)^gamma_init,
 * infall + rotation; cells through the hybrid-EOS prim_to_cons and
 * enforce_floors.  f = {rho, mx, my, mz, E, Bx_f, By_f, Bz_f} in the 3D
 * reference layouts (cells Nx*Ny*Nz, Bx_f (Nx+1)*Ny*Nz, By_f Nx*(Ny+1)*Nz,
 * Bz_f Nx*Ny*(Nz+1), x fastest). */
int cc_ic_mhd3d_reference(const cc_mhd3d_params* p, const cc_mhd3d_ic_knobs* k, double* const* f);

/* The Euler/HLLC main()'s IC, init_random_blob (euler2d_gravity_hllc.cpp:574-642):
 * std::mt19937(42), per cell two uniform(0,1) draws (density and pressure
 * noise) then two uniform(-1,1) draws (velocity); Gaussian density bump.
 * f = {rho, mx, my, E}. */
int cc_ic_euler2d_random_blob(const cc_euler2d_params* p, double* const* f);

/* The Navier-Stokes main()'s collapse IC (navier_stokes_2d_hllc_poisson.cpp:627-700):
 * std::mt19937(p->seed) + std::normal_distribution<double>(0, 1), per cell
 * (j outer, i inner) one draw of density noise then two of velocity;
 * rho = 1 + exp(-r^2 / (2 sigma^2)) + 0.01 N, sigma = 0.1 min(Lx, Ly),
 * P = 0.05, u, v = 0.05 sqrt(gamma P0) N; cells through prim_to_cons
 * (NS:134-145).  f = {rho, mx, my, E}, Nx*Ny doubles each. */
int cc_ic_ns2d_collapse(const cc_ns2d_params* p, double* const* f);

#ifdef __cplusplus
}
#endif

#endif /* CC_IC_H */
