// Host-side initial conditions for the 2D MHD solver (the drop-in main()s and
// the benchmark workloads).  All write the reference layouts (FP64):
// f = {rho, mx, my, mz, E, Bz, Bx_f, By_f}.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "../../include/cc_ic.h"

namespace {

double vmaxd(double a, double b) { return (a < b) ? b : a; }
double vmind(double a, double b) { return (b < a) ? b : a; }
int wrapi(int i, int n) { int r = i % n; return (r < 0) ? r + n : r; }
int clampi(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }

struct Grid {
    const cc_mhd2d_params* p;
    int nx, ny;
    double dx, dy;
    explicit Grid(const cc_mhd2d_params* pp) : p(pp), nx(pp->Nx), ny(pp->Ny) {
        dx = (p->x1 - p->x0) / nx;
        dy = (p->y1 - p->y0) / ny;
    }
    double xc(int i) const { return p->x0 + (i + 0.5) * dx; }
    double yc(int j) const { return p->y0 + (j + 0.5) * dy; }
    // corner potential index with the reference's wrap rule (M2:963-967)
    size_t az(int ic, int jc) const {
        ic = p->periodic_x ? wrapi(ic, nx + 1) : clampi(ic, 0, nx);
        jc = p->periodic_y ? wrapi(jc, ny + 1) : clampi(jc, 0, ny);
        return (size_t)jc * (nx + 1) + ic;
    }
    double bx_cc(const double* bxf, int i, int j) const {
        return 0.5 * (bxf[(size_t)j * (nx + 1) + i] + bxf[(size_t)j * (nx + 1) + i + 1]);
    }
    double by_cc(const double* byf, int i, int j) const {
        return 0.5 * (byf[(size_t)j * nx + i] + byf[(size_t)(j + 1) * nx + i]);
    }
};

// face B from a corner vector potential (M2:992-1006)
void faces_from_Az(const Grid& g, const std::vector<double>& Az, double* bxf, double* byf) {
    for (int j = 0; j < g.ny; ++j)
        for (int i = 0; i <= g.nx; ++i)
            bxf[(size_t)j * (g.nx + 1) + i] = (Az[g.az(i, j + 1)] - Az[g.az(i, j)]) / g.dy;
    for (int j = 0; j <= g.ny; ++j)
        for (int i = 0; i < g.nx; ++i)
            byf[(size_t)j * g.nx + i] = -(Az[g.az(i + 1, j)] - Az[g.az(i, j)]) / g.dx;
}

// prim_to_cons (M2:137-146) then enforce_floors (M2:114-124) into cell q
void set_cell(const cc_mhd2d_params* p, double* const* f, size_t q, double rho, double u, double v, double w, double P,
              double Bx, double By, double Bz) {
    const double gm1 = p->gamma - 1.0;
    double r = vmaxd(rho, p->floor_rho);
    double mx = r * u, my = r * v, mz = r * w;
    double kin = 0.5 * r * (u * u + v * v + w * w);
    double mag = 0.5 * (Bx * Bx + By * By + Bz * Bz);
    double E = kin + mag + P / gm1;
    // enforce_floors
    r = vmaxd(r, p->floor_rho);
    double uu = mx / r, vv = my / r, ww = mz / r;
    double k2 = 0.5 * r * (uu * uu + vv * vv + ww * ww);
    double m2 = 0.5 * (Bx * Bx + By * By + Bz * Bz);
    double Pf = gm1 * (E - k2 - m2);
    if (Pf < p->floor_P) E = k2 + m2 + p->floor_P / gm1;
    f[0][q] = r; f[1][q] = mx; f[2][q] = my; f[3][q] = mz; f[4][q] = E; f[5][q] = Bz;
}

bool valid(const cc_mhd2d_params* p, double* const* f) {
    if (!p || !f || p->Nx < 2 || p->Ny < 2) return false;
    for (int k = 0; k < 8; k++)
        if (!f[k]) return false;
    return true;
}

}  // namespace

extern "C" {

void cc_mhd2d_ic_knobs_default(cc_mhd2d_ic_knobs* k) {
    if (!k) return;
    k->rho_bg = 1.0; k->rho_core = 20.0; k->r_core = 0.12; k->r_edge = 0.02; k->P0 = 0.15;
    k->vin = 1.25; k->rot_omega = 1.0; k->B0x = 0.15; k->Bshear = 0.05; k->gamma_eff = 1.05;
}

int cc_ic_mhd2d_reference(const cc_mhd2d_params* p, const cc_mhd2d_ic_knobs* k, double* const* f) {
    if (!valid(p, f) || !k) return -1;
    Grid g(p);
    const int nx = g.nx, ny = g.ny;
    const double cx = 0.5 * (p->x0 + p->x1), cy = 0.5 * (p->y0 + p->y1);
    std::vector<double> Az((size_t)(nx + 1) * (ny + 1), 0.0);
    for (int jc = 0; jc <= ny; ++jc)
        for (int ic = 0; ic <= nx; ++ic) {
            const double X = p->x0 + ic * g.dx, Y = p->y0 + jc * g.dy;
            const double rx = X - cx, ry = Y - cy;
            const double r = std::sqrt(rx * rx + ry * ry) + 1e-14;
            const double s = (r - k->r_core) / vmaxd(k->r_edge, 1e-12);
            const double shape = 0.5 * (1.0 - std::tanh(s));
            const double base = k->B0x * (Y - p->y0);
            const double Lx = p->x1 - p->x0;
            const double pert = (k->Bshear * k->r_core) * shape * std::sin(2.0 * M_PI * (X - p->x0) / Lx);
            Az[g.az(ic, jc)] = base + pert;
        }
    faces_from_Az(g, Az, f[6], f[7]);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const double X = g.xc(i), Y = g.yc(j);
            const double rx = X - cx, ry = Y - cy;
            const double r = std::sqrt(rx * rx + ry * ry) + 1e-14;
            const double s = (r - k->r_core) / vmaxd(k->r_edge, 1e-12);
            const double shape = 0.5 * (1.0 - std::tanh(s));
            const double rho = k->rho_bg + (k->rho_core - k->rho_bg) * shape;
            const double P = k->P0 * std::pow(rho / vmaxd(k->rho_bg, 1e-12), k->gamma_eff);
            const double vr = -k->vin * (vmind(r / k->r_core, 1.0)) * shape;
            const double vphi = k->rot_omega * r * shape;
            const double erx = rx / r, ery = ry / r;
            const double u = vr * erx + vphi * (-ery);
            const double v = vr * ery + vphi * erx;
            set_cell(p, f, (size_t)j * nx + i, rho, u, v, 0.0, P, g.bx_cc(f[6], i, j), g.by_cc(f[7], i, j), 0.0);
        }
    return 0;
}

int cc_ic_mhd2d_collapse(const cc_mhd2d_params* p, double core_amp, double core_width, double noise, uint32_t seed,
                         double Bx0, double p0, double p_exponent, double* const* f) {
    if (!valid(p, f)) return -1;
    Grid g(p);
    const int nx = g.nx, ny = g.ny;
    const double cx = 0.5 * (p->x0 + p->x1), cy = 0.5 * (p->y0 + p->y1);
    for (size_t q = 0; q < (size_t)(nx + 1) * ny; q++) f[6][q] = Bx0;
    for (size_t q = 0; q < (size_t)nx * (ny + 1); q++) f[7][q] = 0.0;
    std::mt19937 rng(seed);
    std::uniform_real_distribution<double> uni(-1.0, 1.0);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const double rx = g.xc(i) - cx, ry = g.yc(j) - cy;
            const double r2 = rx * rx + ry * ry;
            const double xi = uni(rng);
            const double rho = (1.0 + core_amp * std::exp(-r2 / (2.0 * core_width * core_width))) * (1.0 + noise * xi);
            const double P = p0 * std::pow(rho, p_exponent);
            set_cell(p, f, (size_t)j * nx + i, rho, 0.0, 0.0, 0.0, P, g.bx_cc(f[6], i, j), g.by_cc(f[7], i, j), 0.0);
        }
    return 0;
}

int cc_ic_mhd2d_orszag_tang(const cc_mhd2d_params* p, double core_amp, double core_width, double* const* f) {
    if (!valid(p, f)) return -1;
    Grid g(p);
    const int nx = g.nx, ny = g.ny;
    const double cx = 0.5 * (p->x0 + p->x1), cy = 0.5 * (p->y0 + p->y1);
    const double B0 = 1.0 / std::sqrt(4.0 * M_PI);
    std::vector<double> Az((size_t)(nx + 1) * (ny + 1), 0.0);
    for (int jc = 0; jc <= ny; ++jc)
        for (int ic = 0; ic <= nx; ++ic) {
            const double X = p->x0 + ic * g.dx, Y = p->y0 + jc * g.dy;
            Az[(size_t)jc * (nx + 1) + ic] = B0 * (std::cos(2.0 * M_PI * Y) / (2.0 * M_PI) + std::cos(4.0 * M_PI * X) / (4.0 * M_PI));
        }
    // faces from the corner potential without wrapping (all corners stored)
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i <= nx; ++i)
            f[6][(size_t)j * (nx + 1) + i] = (Az[(size_t)(j + 1) * (nx + 1) + i] - Az[(size_t)j * (nx + 1) + i]) / g.dy;
    for (int j = 0; j <= ny; ++j)
        for (int i = 0; i < nx; ++i)
            f[7][(size_t)j * nx + i] = -(Az[(size_t)j * (nx + 1) + i + 1] - Az[(size_t)j * (nx + 1) + i]) / g.dx;
    const double rho0 = 25.0 / (36.0 * M_PI), P0 = 5.0 / (12.0 * M_PI);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const double X = g.xc(i), Y = g.yc(j);
            const double rx = X - cx, ry = Y - cy;
            const double rho = rho0 + core_amp * std::exp(-(rx * rx + ry * ry) / (2.0 * core_width * core_width));
            const double u = -std::sin(2.0 * M_PI * Y), v = std::sin(2.0 * M_PI * X);
            set_cell(p, f, (size_t)j * nx + i, rho, u, v, 0.0, P0, g.bx_cc(f[6], i, j), g.by_cc(f[7], i, j), 0.0);
        }
    return 0;
}

int cc_ic_euler2d_random_blob(const cc_euler2d_params* p, double* const* f) {
    if (!p || !f || p->Nx < 1 || p->Ny < 1 || !f[0] || !f[1] || !f[2] || !f[3]) return -1;
    const int nx = p->Nx, ny = p->Ny;
    const double dx = (p->x1 - p->x0) / nx, dy = (p->y1 - p->y0) / ny;
    std::mt19937 rng(42);
    std::uniform_real_distribution<double> uni01(0.0, 1.0);
    std::uniform_real_distribution<double> uniV(-1.0, 1.0);
    const double rho0 = 1.0, P0 = 1.0, amp_rho = 0.10, amp_P = 0.10, vmax = 0.05;
    const double xc = 0.5 * (p->x0 + p->x1), yc = 0.5 * (p->y0 + p->y1);
    const double sigma = 0.08, bump_amp = 0.5;
    const double gm1 = p->gamma - 1.0;
    for (int j = 0; j < ny; ++j) {
        const double y = p->y0 + (j + 0.5) * dy;
        for (int i = 0; i < nx; ++i) {
            const double x = p->x0 + (i + 0.5) * dx;
            const size_t k = (size_t)j * nx + i;
            const double fr = 2.0 * uni01(rng) - 1.0;
            const double fp = 2.0 * uni01(rng) - 1.0;
            double rho = rho0 * (1.0 + amp_rho * fr);
            double P = P0 * (1.0 + amp_P * fp);
            const double rx = x - xc, ry = y - yc, r2 = rx * rx + ry * ry;
            rho += bump_amp * rho0 * std::exp(-r2 / (2.0 * sigma * sigma));
            const double u = vmax * uniV(rng);
            const double v = vmax * uniV(rng);
            rho = vmaxd(rho, p->floor_rho);
            P = vmaxd(P, p->floor_P);
            double r = rho, mx = rho * u, my = rho * v, E = P / gm1 + 0.5 * rho * (u * u + v * v);
            // enforce_floors (EH:62-72)
            r = vmaxd(r, p->floor_rho);
            const double uu = mx / r, vv = my / r, kin = 0.5 * r * (uu * uu + vv * vv);
            if (gm1 * (E - kin) < p->floor_P) E = kin + p->floor_P / gm1;
            f[0][k] = r; f[1][k] = mx; f[2][k] = my; f[3][k] = E;
        }
    }
    return 0;
}

int cc_ic_ns2d_collapse(const cc_ns2d_params* p, double* const* f) {
    if (!p || !f || p->Nx < 1 || p->Ny < 1 || !f[0] || !f[1] || !f[2] || !f[3]) return -1;
    const int nx = p->Nx, ny = p->Ny;
    const double Lx = p->x1 - p->x0, Ly = p->y1 - p->y0;
    const double dx = Lx / nx, dy = Ly / ny;
    std::mt19937 rng(p->seed);
    std::normal_distribution<double> gauss(0.0, 1.0);
    // background, Gaussian overdensity, 1% density noise, Mach-0.05 velocity noise (NS:638-659)
    const double rho0 = 1.0, P0 = 0.05, A = 1, sigma = 0.10 * vmind(Lx, Ly), Arho = 0.01;
    const double a0 = std::sqrt(p->gamma * P0 / rho0), Mach0 = 0.05, vamp = Mach0 * a0;
    const double xc = 0.5 * (p->x0 + p->x1), yc = 0.5 * (p->y0 + p->y1);
    for (int j = 0; j < ny; ++j) {
        const double y = p->y0 + (j + 0.5) * dy;
        for (int i = 0; i < nx; ++i) {
            const double x = p->x0 + (i + 0.5) * dx;
            const double rx = x - xc, ry = y - yc, r2 = rx * rx + ry * ry;
            const double bump = A * std::exp(-0.5 * r2 / (sigma * sigma));
            const double noise = Arho * gauss(rng);
            const double d0 = vmaxd(rho0 * (1.0 + bump + noise), p->floor_rho);
            const double P = vmaxd(P0, p->floor_P);
            const double u = vamp * gauss(rng);
            const double v = vamp * gauss(rng);
            // prim_to_cons (NS:134-145)
            const double d = vmaxd(d0, p->floor_rho), Pc = vmaxd(P, p->floor_P);
            const size_t k = (size_t)j * nx + i;
            f[0][k] = d;
            f[1][k] = d * u;
            f[2][k] = d * v;
            f[3][k] = Pc / (p->gamma - 1.0) + 0.5 * d * (u * u + v * v);
        }
    }
    return 0;
}

}  // extern "C"
