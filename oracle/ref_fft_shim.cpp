// ORACLE / TEST INFRASTRUCTURE ONLY.  Compiles navier_stokes_2d_hllc_poisson.cpp
// in place (via -I, never copied) inside a private namespace and exports its
// spectral Poisson solve and its Navier-Stokes step functions through a C ABI:
//   solve_poisson_periodic_fft  NS:285-328 (fft1d NS:152-177, fft2d NS:179-195)
//   compute_gravity_accel       NS:330-360
//   compute_rhs                 NS:363-518 (hllc_x/hllc_y, viscous stress, gravity source)
//   compute_dt                  NS:521-546
#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdlib>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>
#include "hdf5.h"

#define main ref_ns_main
namespace refns {
#include "navier_stokes_2d_hllc_poisson.cpp"
}
#undef main

extern "C" {

int ref_fft_poisson(int Nx, int Ny, double x0, double x1, double y0, double y1, double G,
                    const double* rho, double* phi) {
    using namespace refns;
    Grid2D g(Nx, Ny, x0, x1, y0, y1);
    Params p; p.G = G;
    std::vector<double> r(rho, rho + (size_t)Nx * Ny), ph;
    solve_poisson_periodic_fft(r, ph, g, p);
    std::copy(ph.begin(), ph.end(), phi);
    return 0;
}

int ref_fft_gravity_accel(int Nx, int Ny, double x0, double x1, double y0, double y1,
                          const double* phi, double* gx, double* gy) {
    using namespace refns;
    Grid2D g(Nx, Ny, x0, x1, y0, y1);
    std::vector<double> ph(phi, phi + (size_t)Nx * Ny), ax, ay;
    compute_gravity_accel(ph, ax, ay, g);
    std::copy(ax.begin(), ax.end(), gx);
    std::copy(ay.begin(), ay.end(), gy);
    return 0;
}

// One 1D transform of the reference (NS:152-177) on interleaved re/im data.
int ref_fft1d(int n, double* reim, int inverse) {
    using namespace refns;
    std::vector<std::complex<double>> a(n);
    for (int i = 0; i < n; i++) a[i] = {reim[2 * i], reim[2 * i + 1]};
    fft1d(a, inverse != 0);
    for (int i = 0; i < n; i++) { reim[2 * i] = a[i].real(); reim[2 * i + 1] = a[i].imag(); }
    return 0;
}

// Navier-Stokes parameters that the step functions read (Params, NS:54-86)
static refns::Params ns_params(double gamma, double floor_rho, double floor_P, int viscosity_on, double mu,
                               double cfl, double cfl_visc, int gravity_on, double G) {
    refns::Params p;
    p.gamma = gamma; p.floor_rho = floor_rho; p.floor_P = floor_P;
    p.viscosity_on = viscosity_on != 0; p.mu = mu; p.cfl = cfl; p.cfl_visc = cfl_visc;
    p.gravity_on = gravity_on != 0; p.G = G;
    return p;
}

// compute_rhs(U) (NS:363-518): f, dU = {rho, mx, my, E}, Nx*Ny each
int ref_ns_rhs(int Nx, int Ny, double x0, double x1, double y0, double y1, double gamma, double floor_rho,
               double floor_P, int viscosity_on, double mu, int gravity_on, double G, const double* const* f,
               double* const* dU) {
    using namespace refns;
    Grid2D g(Nx, Ny, x0, x1, y0, y1);
    const Params p = ns_params(gamma, floor_rho, floor_P, viscosity_on, mu, 0.35, 0.05, gravity_on, G);
    const size_t n = (size_t)Nx * Ny;
    std::vector<U4> U(n), R;
    for (size_t q = 0; q < n; q++) U[q] = U4{f[0][q], f[1][q], f[2][q], f[3][q]};
    compute_rhs(U, R, g, p);
    for (size_t q = 0; q < n; q++) {
        dU[0][q] = R[q].d; dU[1][q] = R[q].mx; dU[2][q] = R[q].my; dU[3][q] = R[q].E;
    }
    return 0;
}

// compute_dt(U) (NS:521-546)
double ref_ns_dt(int Nx, int Ny, double x0, double x1, double y0, double y1, double gamma, double cfl,
                 double floor_rho, double floor_P, int viscosity_on, double mu, double cfl_visc,
                 const double* const* f) {
    using namespace refns;
    Grid2D g(Nx, Ny, x0, x1, y0, y1);
    const Params p = ns_params(gamma, floor_rho, floor_P, viscosity_on, mu, cfl, cfl_visc, 1, 10.0);
    const size_t n = (size_t)Nx * Ny;
    std::vector<U4> U(n);
    for (size_t q = 0; q < n; q++) U[q] = U4{f[0][q], f[1][q], f[2][q], f[3][q]};
    return compute_dt(U, g, p);
}

}  // extern "C"
