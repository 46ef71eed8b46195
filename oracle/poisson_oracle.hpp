// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// CPU restatements of the periodic/outflow Poisson solves used for self-gravity:
//   sor_lexicographic  M2:178-237 (fixed sweeps) and EH:288-386 (residual tolerance)
//   sor_red_black      the GPU ordering of the same SOR update (red cells (i+j) even,
//                      then black), mean removed after each full sweep, residual
//                      max|lap(phi)-rhs| of the current iterate checked after it
//   fft_periodic       NS:152-195 (radix-2 FFT, twiddles by recurrence) and NS:285-328
//   gravity_from_phi   M2:225-235 (g = -central difference of phi)
// All in double, whatever the caller's state type.
#pragma once
#include <cmath>
#include <complex>
#include <vector>

#include "oracle_common.hpp"

namespace cco {

struct PoissonSpec {
    int nx, ny;
    bool px, py;
    double dx, dy;
    double G;
    double omega;
    int max_iter;
    double tol;          // <= 0: run exactly max_iter sweeps
    bool floor_density;  // EH floors rho before the solve (EH:312)
    double floor_rho;
    double Lx, Ly;       // box lengths for the spectral wavenumbers
};

struct PoissonResult {
    int iters = 0;
    double residual = 0.0;
};

inline size_t pidx(const PoissonSpec& s, int i, int j) {
    Axis ax{s.nx, s.px}, ay{s.ny, s.py};
    return (size_t)ay.cell(j) * s.nx + ax.cell(i);
}

// rhs = 4 pi G (rho - mean(rho)), mean by a sequential sum (M2:187-194)
inline std::vector<double> poisson_rhs(const PoissonSpec& s, const std::vector<double>& rho_in) {
    const size_t N = (size_t)s.nx * s.ny;
    std::vector<double> rho(rho_in.begin(), rho_in.begin() + N);
    if (s.floor_density)
        for (auto& r : rho) r = vmax(r, s.floor_rho);
    double mean = 0.0;
    for (double r : rho) mean += r;
    mean /= (double)N;
    std::vector<double> rhs(N);
    for (size_t q = 0; q < N; q++) rhs[q] = 4.0 * M_PI * s.G * (rho[q] - mean);
    return rhs;
}

inline void remove_mean(std::vector<double>& phi) {
    double m = 0.0;
    for (double v : phi) m += v;
    m /= (double)phi.size();
    for (double& v : phi) v -= m;
}

inline double residual_max(const PoissonSpec& s, const std::vector<double>& phi, const std::vector<double>& rhs) {
    const double idx2 = 1.0 / (s.dx * s.dx), idy2 = 1.0 / (s.dy * s.dy);
    double r = 0.0;
    for (int j = 0; j < s.ny; j++)
        for (int i = 0; i < s.nx; i++) {
            size_t k = (size_t)j * s.nx + i;
            double c = phi[k];
            double lap = (phi[pidx(s, i + 1, j)] - 2.0 * c + phi[pidx(s, i - 1, j)]) * idx2 +
                         (phi[pidx(s, i, j + 1)] - 2.0 * c + phi[pidx(s, i, j - 1)]) * idy2;
            r = vmax(r, std::abs(lap - rhs[k]));
        }
    return r;
}

// Lexicographic SOR.  tol <= 0: M2:207-223 (fixed sweeps).  tol > 0: EH:335-368,
// the residual taken inside the sweep from the just-updated value.
inline PoissonResult sor_lexicographic(const PoissonSpec& s, const std::vector<double>& rhs, std::vector<double>& phi) {
    const double idx2 = 1.0 / (s.dx * s.dx), idy2 = 1.0 / (s.dy * s.dy);
    const double denom = 2.0 * (idx2 + idy2);
    phi.assign((size_t)s.nx * s.ny, 0.0);
    PoissonResult out;
    for (int it = 0; it < s.max_iter; ++it) {
        double max_res = 0.0;
        for (int j = 0; j < s.ny; j++)
            for (int i = 0; i < s.nx; i++) {
                size_t k = (size_t)j * s.nx + i;
                double pE = phi[pidx(s, i + 1, j)], pW = phi[pidx(s, i - 1, j)];
                double pN = phi[pidx(s, i, j + 1)], pS = phi[pidx(s, i, j - 1)];
                double pn = ((pE + pW) * idx2 + (pN + pS) * idy2 - rhs[k]) / denom;
                phi[k] += s.omega * (pn - phi[k]);
                if (s.tol > 0.0) {
                    double lap = (pE - 2.0 * phi[k] + pW) * idx2 + (pN - 2.0 * phi[k] + pS) * idy2;
                    max_res = vmax(max_res, std::abs(lap - rhs[k]));
                }
            }
        remove_mean(phi);
        out.iters = it + 1;
        out.residual = max_res;
        if (s.tol > 0.0 && max_res < s.tol) break;
    }
    return out;
}

// Red-black SOR: the parallel ordering the GPU uses.  Within one colour no
// cell reads another cell of the same colour (grids with an even periodic
// extent, or any outflow extent), so the colour update is order-free.
inline PoissonResult sor_red_black(const PoissonSpec& s, const std::vector<double>& rhs, std::vector<double>& phi) {
    const double idx2 = 1.0 / (s.dx * s.dx), idy2 = 1.0 / (s.dy * s.dy);
    const double denom = 2.0 * (idx2 + idy2);
    phi.assign((size_t)s.nx * s.ny, 0.0);
    PoissonResult out;
    for (int it = 0; it < s.max_iter; ++it) {
        for (int colour = 0; colour < 2; ++colour)
            for (int j = 0; j < s.ny; j++)
                for (int i = (j + colour) & 1; i < s.nx; i += 2) {
                    size_t k = (size_t)j * s.nx + i;
                    double pE = phi[pidx(s, i + 1, j)], pW = phi[pidx(s, i - 1, j)];
                    double pN = phi[pidx(s, i, j + 1)], pS = phi[pidx(s, i, j - 1)];
                    double pn = ((pE + pW) * idx2 + (pN + pS) * idy2 - rhs[k]) / denom;
                    phi[k] += s.omega * (pn - phi[k]);
                }
        remove_mean(phi);
        out.iters = it + 1;
        if (s.tol > 0.0) {
            out.residual = residual_max(s, phi, rhs);
            if (out.residual < s.tol) break;
        }
    }
    if (!(s.tol > 0.0)) out.residual = residual_max(s, phi, rhs);
    return out;
}

// Twiddles of one radix-2 pass of length len, built by the reference's
// recurrence w_{j+1} = w_j * wlen (NS:161-171).
inline std::vector<std::complex<double>> fft_twiddles(int len, bool inverse) {
    const double ang = 2.0 * M_PI / len * (inverse ? +1.0 : -1.0);
    std::complex<double> wlen(std::cos(ang), std::sin(ang)), w(1.0, 0.0);
    std::vector<std::complex<double>> t(len / 2);
    for (int j = 0; j < len / 2; j++) { t[j] = w; w *= wlen; }
    return t;
}

// In-place radix-2 decimation-in-time FFT (NS:152-177).
inline void fft_1d(std::vector<std::complex<double>>& a, bool inverse) {
    const int n = (int)a.size();
    for (int i = 1, j = 0; i < n; i++) {
        int bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) std::swap(a[i], a[j]);
    }
    for (int len = 2; len <= n; len <<= 1) {
        std::vector<std::complex<double>> tw = fft_twiddles(len, inverse);
        for (int i = 0; i < n; i += len)
            for (int j = 0; j < len / 2; j++) {
                std::complex<double> u = a[i + j], v = a[i + j + len / 2] * tw[j];
                a[i + j] = u + v;
                a[i + j + len / 2] = u - v;
            }
    }
    if (inverse)
        for (auto& z : a) z /= (double)n;
}

// rows then columns, for both directions (NS:179-195)
inline void fft_2d(std::vector<std::complex<double>>& A, int nx, int ny, bool inverse) {
    std::vector<std::complex<double>> line;
    for (int j = 0; j < ny; j++) {
        line.assign(A.begin() + (size_t)j * nx, A.begin() + (size_t)(j + 1) * nx);
        fft_1d(line, inverse);
        std::copy(line.begin(), line.end(), A.begin() + (size_t)j * nx);
    }
    line.resize(ny);
    for (int i = 0; i < nx; i++) {
        for (int j = 0; j < ny; j++) line[j] = A[(size_t)j * nx + i];
        fft_1d(line, inverse);
        for (int j = 0; j < ny; j++) A[(size_t)j * nx + i] = line[j];
    }
}

// Spectral periodic solve phi_k = -4 pi G rho_k / |k|^2 (NS:285-328).
inline void fft_periodic(const PoissonSpec& s, const std::vector<double>& rho, std::vector<double>& phi) {
    const int nx = s.nx, ny = s.ny;
    const size_t N = (size_t)nx * ny;
    double mean = 0.0;
    for (size_t q = 0; q < N; q++) mean += rho[q];
    mean /= (double)N;
    std::vector<std::complex<double>> A(N);
    for (size_t q = 0; q < N; q++) A[q] = std::complex<double>(rho[q] - mean, 0.0);
    fft_2d(A, nx, ny, false);
    const double two_pi = 2.0 * M_PI;
    for (int j = 0; j < ny; j++) {
        int nj = (j <= ny / 2) ? j : j - ny;
        double ky = two_pi * (double)nj / s.Ly;
        for (int i = 0; i < nx; i++) {
            int ni = (i <= nx / 2) ? i : i - nx;
            double kx = two_pi * (double)ni / s.Lx;
            double k2 = kx * kx + ky * ky;
            size_t q = (size_t)j * nx + i;
            if (k2 == 0.0) A[q] = 0.0;
            else A[q] *= (-(4.0 * M_PI * s.G) / k2);
        }
    }
    fft_2d(A, nx, ny, true);
    phi.resize(N);
    for (size_t q = 0; q < N; q++) phi[q] = A[q].real();
}

// ---------------------------------------------------------------------------
// Direct solve of the discrete problem the SOR iterates towards (the
// library's batched-ensemble Poisson): 5-point Laplacian with the solver's
// boundary rule (clamp = mirrored ghost, periodic = wrap), zero-mean solution.
//   1. x transform by a dense orthonormal eigenbasis of the x second
//      difference: DCT-II for clamp, discrete Hartley (cas) for periodic;
//   2. per x wavenumber k, the y system (Dyy + lam_x[k]) u = r: Thomas
//      (clamp y), Sherman-Morrison cyclic Thomas (periodic y), and for k = 0
//      (singular) the cumulative-flux solution with its mean removed;
//   3. inverse x transform.
// Every multiply-add the library fuses is written as std::fma here, in the
// same order, so that the double result matches the library bit for bit.
// ---------------------------------------------------------------------------

// Row k of `basis` (n x n) is the k-th orthonormal eigenvector; lam[k] its
// eigenvalue of (u[i+1] - 2u[i] + u[i-1]) / d^2 under the boundary rule.
inline void direct_basis(int n, bool periodic, double d, std::vector<double>& basis, std::vector<double>& lam) {
    basis.assign((size_t)n * n, 0.0);
    lam.assign(n, 0.0);
    for (int k = 0; k < n; k++) {
        double sn;
        if (periodic) {
            const double sc = 1.0 / std::sqrt((double)n);
            for (int i = 0; i < n; i++) {
                const double arg = 2.0 * M_PI * (double)(((long long)k * i) % n) / (double)n;
                basis[(size_t)k * n + i] = (std::cos(arg) + std::sin(arg)) * sc;
            }
            sn = std::sin(M_PI * (double)k / (double)n);
        } else {
            const double sc = std::sqrt((k == 0 ? 1.0 : 2.0) / (double)n);
            for (int i = 0; i < n; i++) {
                const double arg = M_PI * (double)((long long)k * (2 * i + 1)) / (double)(2 * n);
                basis[(size_t)k * n + i] = sc * std::cos(arg);
            }
            sn = std::sin(M_PI * (double)k / (double)(2 * n));
        }
        lam[k] = -4.0 * sn * sn / (d * d);
    }
}

// Density mean in the batched reduction order: 32 x 8 cell tiles in row-major
// tile order; inside a tile a warp holds one row of 32 cells, the lanes are
// summed by a shuffle-down tree (offsets 16..1), then the 8 warp sums by the
// same tree (absent lanes 0.0).  The tile sums are folded by 32 lanes (lane
// l: tiles l, l+32, ... in order) and the lane values by the same tree.
inline double batch_tile_mean(int nx, int ny, const std::vector<double>& rho) {
    const int tx_n = (nx + 31) / 32, ty_n = (ny + 7) / 8;
    double lane[32];
    for (int l = 0; l < 32; l++) lane[l] = 0.0;
    int t = 0;
    for (int ty = 0; ty < ty_n; ty++)
        for (int tx = 0; tx < tx_n; tx++, t++) {
            double w[32];
            for (int r = 0; r < 32; r++) w[r] = 0.0;
            for (int r = 0; r < 8; r++) {
                double v[32];
                for (int l = 0; l < 32; l++) {
                    const int i = tx * 32 + l, j = ty * 8 + r;
                    v[l] = (i < nx && j < ny) ? rho[(size_t)j * nx + i] : 0.0;
                }
                for (int o = 16; o > 0; o >>= 1)
                    for (int l = 0; l < o; l++) v[l] = v[l] + v[l + o];
                w[r] = v[0];
            }
            for (int o = 16; o > 0; o >>= 1)
                for (int l = 0; l < o; l++) w[l] = w[l] + w[l + o];
            lane[t % 32] = lane[t % 32] + w[0];
        }
    for (int o = 16; o > 0; o >>= 1)
        for (int l = 0; l < o; l++) lane[l] = lane[l] + lane[l + o];
    return lane[0] / ((double)nx * (double)ny);
}

// Factors of the y system (Dyy + lam) u = r for one x wavenumber, set up
// once per grid: m_j = b_j - a cp_{j-1} (fma), inv_j = 1/m_j, cp_j = a inv_j;
// the clamp rule's end rows have b = lam - a.  Periodic y (cyclic system):
// Sherman-Morrison with gamma = -b, u = (gamma, 0.., a), v = (1, 0.., a/gamma);
// T' has b - gamma at row 0 and b - a*a/gamma at row n-1; z = T'^-1 u and
// fden = 1 / (1 + v.z) are part of the factors.
struct YFactors {
    std::vector<double> cp, inv, z;
    double fden = 0.0;
};

inline YFactors direct_yfactors(int n, bool py, double a, double lam) {
    YFactors f;
    f.cp.assign(n, 0.0);
    f.inv.assign(n, 0.0);
    const double b = std::fma(-2.0, a, lam);
    const double gam = -b;
    const double bE = py ? b - gam : lam - a;           // row 0
    const double bL = py ? b - a * a / gam : lam - a;   // row n-1
    double cprev = 0.0;
    for (int j = 0; j < n; j++) {
        const double bj = (j == 0) ? bE : (j == n - 1 ? bL : b);
        const double m = (j == 0) ? bj : std::fma(-a, cprev, bj);
        f.inv[j] = 1.0 / m;
        cprev = a * f.inv[j];
        f.cp[j] = cprev;
    }
    if (py) {
        f.z.assign(n, 0.0);
        for (int j = 0; j < n; j++) {
            const double zr = (j == 0) ? gam : (j == n - 1 ? a : 0.0);
            f.z[j] = (j == 0) ? zr * f.inv[0] : std::fma(-a, f.z[j - 1], zr) * f.inv[j];
        }
        for (int j = n - 2; j >= 0; j--) f.z[j] = std::fma(-f.cp[j], f.z[j + 1], f.z[j]);
        f.fden = 1.0 / (1.0 + std::fma(a / gam, f.z[n - 1], f.z[0]));
    }
    return f;
}

// One y system for x wavenumber k (column col of the ny x nx array u, solved in place).
inline void direct_ysolve(int nx, int ny, bool py, double ay, double dy2, double lam, bool singular, int col,
                          std::vector<double>& u) {
    auto at = [&](int j) -> double& { return u[(size_t)j * nx + col]; };
    const int n = ny;
    if (singular) {
        // flux G_j = a (u_{j+1} - u_j) = G_{j-1} + r_j; clamp: G_{-1} = 0;
        // periodic: G_{-1} = -(1/n) sum_j S_j with S_j the running sum of r
        double g0 = 0.0;
        if (py) {
            double S = 0.0, SS = 0.0;
            for (int j = 0; j < n; j++) { S = S + at(j); SS = SS + S; }
            g0 = -(SS / (double)n);
        }
        double G = g0, prev = 0.0;
        std::vector<double> out(n);
        out[0] = 0.0;
        for (int j = 0; j + 1 < n; j++) {
            G = G + at(j);
            prev = std::fma(dy2, G, prev);
            out[j + 1] = prev;
        }
        double m = 0.0;
        for (int j = 0; j < n; j++) m = m + out[j];
        m = m / (double)n;
        for (int j = 0; j < n; j++) at(j) = out[j] - m;
        return;
    }
    const double a = ay;
    const YFactors f = direct_yfactors(n, py, a, lam);
    at(0) = at(0) * f.inv[0];
    for (int j = 1; j < n; j++) at(j) = std::fma(-a, at(j - 1), at(j)) * f.inv[j];
    for (int j = n - 2; j >= 0; j--) at(j) = std::fma(-f.cp[j], at(j + 1), at(j));
    if (!py) return;
    const double gam = -std::fma(-2.0, a, lam);
    const double fac = std::fma(a / gam, at(n - 1), at(0)) * f.fden;
    for (int j = 0; j < n; j++) at(j) = std::fma(-fac, f.z[j], at(j));
}

// phi solving lap(phi) = rhs (ny x nx row-major), zero mean.
inline void direct_solve(const PoissonSpec& s, const std::vector<double>& rhs, std::vector<double>& phi) {
    const int nx = s.nx, ny = s.ny;
    std::vector<double> tx, lam;
    direct_basis(nx, s.px, s.dx, tx, lam);
    std::vector<double> u((size_t)nx * ny);
    // u[j][k] = sum_i rhs[j][i] tx[k][i], i ascending
    for (int j = 0; j < ny; j++)
        for (int k = 0; k < nx; k++) {
            double acc = 0.0;
            for (int i = 0; i < nx; i++) acc = std::fma(rhs[(size_t)j * nx + i], tx[(size_t)k * nx + i], acc);
            u[(size_t)j * nx + k] = acc;
        }
    const double ay = 1.0 / (s.dy * s.dy), dy2 = s.dy * s.dy;
    for (int k = 0; k < nx; k++) direct_ysolve(nx, ny, s.py, ay, dy2, lam[k], k == 0, k, u);
    phi.assign((size_t)nx * ny, 0.0);
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            double acc = 0.0;
            for (int k = 0; k < nx; k++) acc = std::fma(u[(size_t)j * nx + k], tx[(size_t)k * nx + i], acc);
            phi[(size_t)j * nx + i] = acc;
        }
}

// rhs of the direct solve: 4 pi G (rho - mean), mean in the batched order
inline std::vector<double> direct_rhs(const PoissonSpec& s, const std::vector<double>& rho) {
    const size_t N = (size_t)s.nx * s.ny;
    const double mean = batch_tile_mean(s.nx, s.ny, rho);
    const double fourpiG = 4.0 * M_PI * s.G;
    std::vector<double> rhs(N);
    for (size_t q = 0; q < N; q++) rhs[q] = fourpiG * (rho[q] - mean);
    return rhs;
}

// g = -grad(phi), central differences with the solver's wrap rule (M2:225-235)
inline void gravity_from_phi(const PoissonSpec& s, const std::vector<double>& phi, std::vector<double>& gx,
                             std::vector<double>& gy) {
    gx.assign((size_t)s.nx * s.ny, 0.0);
    gy.assign((size_t)s.nx * s.ny, 0.0);
    for (int j = 0; j < s.ny; j++)
        for (int i = 0; i < s.nx; i++) {
            size_t k = (size_t)j * s.nx + i;
            gx[k] = -(phi[pidx(s, i + 1, j)] - phi[pidx(s, i - 1, j)]) / (2.0 * s.dx);
            gy[k] = -(phi[pidx(s, i, j + 1)] - phi[pidx(s, i, j - 1)]) / (2.0 * s.dy);
        }
}

}  // namespace cco
