// ORACLE / TEST INFRASTRUCTURE ONLY.  Compiles gravity_enclosed.h in place (via
// -I, never copied) and exports its shell-binned enclosed-mass gravity
// (gravity_accel_from_enclosed_mass, gravity_enclosed.h:18-96) through a C
// ABI.  The header expects its includer to define Params, Grid2D, U2D and
// idx(); the definitions below carry just the fields it reads, with cell
// centres x0 + (i + 1/2) dx, y0 + (j + 1/2) dy.  The standard headers that the
// header includes come first, so that its includes inside the namespace are no-ops.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <vector>

namespace refge {
struct Params {
    bool gravity_on = true;
    double G = 1.0, softening = 1e-4, xc = 0.5, yc = 0.5, floor_rho = 1e-12, gamma = 1.4, floor_P = 1e-12;
    int Nr_bins = 512;
};
struct Grid2D {
    int Nx = 0, Ny = 0;
    double dx = 0.0, dy = 0.0;
    std::vector<double> x, y;
};
struct U2D { std::vector<double> rho, mx, my, E; };
static inline size_t idx(int i, int j, int Nx) { return (size_t)j * (size_t)Nx + (size_t)i; }
#include "gravity_enclosed.h"
}  // namespace refge

extern "C" int ref_ge_gravity(int Nx, int Ny, double x0, double x1, double y0, double y1, double G, double softening,
                              int Nr_bins, double xc, double yc, double floor_rho, const double* rho, double* gx,
                              double* gy) {
    using namespace refge;
    Grid2D g;
    g.Nx = Nx; g.Ny = Ny;
    g.dx = (x1 - x0) / Nx; g.dy = (y1 - y0) / Ny;
    for (int i = 0; i < Nx; i++) g.x.push_back(x0 + (i + 0.5) * g.dx);
    for (int j = 0; j < Ny; j++) g.y.push_back(y0 + (j + 0.5) * g.dy);
    Params p;
    p.G = G; p.softening = softening; p.Nr_bins = Nr_bins; p.xc = xc; p.yc = yc; p.floor_rho = floor_rho;
    U2D U;
    U.rho.assign(rho, rho + (size_t)Nx * Ny);
    std::vector<double> ax, ay;
    gravity_accel_from_enclosed_mass(U, g, p, ax, ay);
    for (size_t q = 0; q < ax.size(); q++) { gx[q] = ax[q]; gy[q] = ay[q]; }
    return 0;
}
