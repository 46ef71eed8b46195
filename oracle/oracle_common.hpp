// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into core_collapse_b200.
//
// CPU restatement of the reference finite-volume step, used by tests/ and by
// bench.py's CPU-baseline leg as the checker.  This header holds the pieces
// shared by the 2D and 3D restatements: std::max/std::min/std::abs with the
// exact semantics the reference relies on, index wrapping, and the MC limiter.
//
// The restatement is templated on the arithmetic type T (double for parity,
// float for precision studies).  Every expression keeps the reference's
// evaluation order so that, compiled without FMA contraction
// (-ffp-contract=off), T=double reproduces the reference bit for bit.
#pragma once
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <vector>

namespace cco {

// std::max(a,b) is (a<b)?b:a and std::min(a,b) is (b<a)?b:a; the NaN
// behaviour of these (first argument wins) matters in compute_dt.
template <class T> inline T vmax(T a, T b) { return (a < b) ? b : a; }
template <class T> inline T vmin(T a, T b) { return (b < a) ? b : a; }

inline int wrap_idx(int i, int n) { int r = i % n; return (r < 0) ? r + n : r; }
inline int clamp_idx(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }

// One axis of the grid: cell indices wrap modulo n (periodic) or clamp to
// [0,n-1]; face indices along the axis wrap modulo n+1 or clamp to [0,n]
// (mhd2d_resistive_hlld_ct_gravity.cpp:241-252).
struct Axis {
    int n;
    bool periodic;
    int cell(int i) const { return periodic ? wrap_idx(i, n) : clamp_idx(i, 0, n - 1); }
    int face(int i) const { return periodic ? wrap_idx(i, n + 1) : clamp_idx(i, 0, n); }
};

// minmod / MC limiter (M2:106-112, M3:106-112, EH:85-92).
template <class T> inline T minmod(T a, T b) {
    if (a * b <= T(0)) return T(0);
    return (std::abs(a) < std::abs(b)) ? a : b;
}
template <class T> inline T mc_slope(T dm, T dp) {
    return minmod(T(0.5) * (dm + dp), minmod(T(2.0) * dm, T(2.0) * dp));
}

}  // namespace cco
