// Host-built twiddle tables of the spectral Poisson solves (2D MHD and
// Navier-Stokes handles).
#pragma once
#include <cmath>
#include <vector>

namespace ccb {

// n-th roots of unity W^e = (cos 2 pi e / n, -sin 2 pi e / n), e < n, for the
// FP32 spectral solve (evaluated in FP64, then rounded)
inline std::vector<float> fft32_roots(int n) {
    std::vector<float> t(2 * (size_t)n);
    for (int e = 0; e < n; e++) {
        const double ang = 2.0 * M_PI * (double)e / (double)n;
        t[2 * (size_t)e] = (float)std::cos(ang);
        t[2 * (size_t)e + 1] = (float)-std::sin(ang);
    }
    return t;
}

// Twiddles of every radix-2 pass of an n-point transform by the reference's
// recurrence w_{j+1} = w_j * wlen (navier_stokes_2d_hllc_poisson.cpp:160-171),
// pass with half-length h stored at [h-1, 2h-1).
inline std::vector<double> twiddle_table(int n, bool inverse) {
    std::vector<double> t(2 * (size_t)(n > 1 ? n - 1 : 1), 0.0);
    for (int len = 2; len <= n; len <<= 1) {
        const double ang = 2.0 * M_PI / len * (inverse ? +1.0 : -1.0);
        const double wr = std::cos(ang), wi = std::sin(ang);
        double cr = 1.0, ci = 0.0;
        const int h = len / 2;
        for (int j = 0; j < h; j++) {
            t[2 * (size_t)(h - 1 + j)] = cr;
            t[2 * (size_t)(h - 1 + j) + 1] = ci;
            const double nr = cr * wr - ci * wi, ni = cr * wi + ci * wr;
            cr = nr; ci = ni;
        }
    }
    return t;
}

}  // namespace ccb
