// ORACLE / TEST INFRASTRUCTURE ONLY.  Compiles navier_stokes_2d_hllc_poisson.cpp
// in place (via -I, never copied) inside a private namespace and exports its
// spectral Poisson solve through a C ABI:
//   solve_poisson_periodic_fft  NS:285-328 (fft1d NS:152-177, fft2d NS:179-195)
//   compute_gravity_accel       NS:330-360
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

}  // extern "C"
