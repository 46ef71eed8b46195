// Device-side helpers shared by every kernel of libcc_b200: min/max with the
// reference's std::max/std::min semantics, index wrapping, deterministic block
// reductions and a bounded grid barrier for persistent kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ccb {

// std::max(a,b) == (a<b)?b:a, std::min(a,b) == (b<a)?b:a.  Kept exactly so
// that branch-sensitive code (floors, limiter, wave-speed bounds) takes the
// same branches as the reference.
template <class T> __host__ __device__ __forceinline__ T vmax(T a, T b) { return (a < b) ? b : a; }
template <class T> __host__ __device__ __forceinline__ T vmin(T a, T b) { return (b < a) ? b : a; }

// The reference's positive guard 1e-300 (a division or square-root floor); FP32
// cannot hold it and its instantiations use 1e-30, a normal FP32 value far
// below every density floor
template <class T> __host__ __device__ constexpr T tiny_pos() { return sizeof(T) == 4 ? T(1e-30f) : T(1e-300); }

__host__ __device__ __forceinline__ int wrap_idx(int i, int n) { int r = i % n; return (r < 0) ? r + n : r; }
__host__ __device__ __forceinline__ int clamp_idx(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }

// One grid axis.  Cell indices wrap modulo n (periodic) or clamp to [0,n-1];
// face indices along the axis wrap modulo n+1 or clamp to [0,n]
// (mhd2d_resistive_hlld_ct_gravity.cpp:241-252).
struct AxisMap {
    int n;
    int periodic;
    __host__ __device__ __forceinline__ int cell(int i) const {
        if (i >= 0 && i < n) return i;
        return periodic ? wrap_idx(i, n) : clamp_idx(i, 0, n - 1);
    }
    __host__ __device__ __forceinline__ int face(int i) const {
        if (i >= 0 && i <= n) return i;
        return periodic ? wrap_idx(i, n + 1) : clamp_idx(i, 0, n);
    }
};

// Deterministic sum over a block: fixed shuffle tree inside each warp, then
// warp partials summed in warp order by warp 0.  Result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh /* >= NT/32 */) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < NT / 32) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// Max over a block of non-negative values (order-free).  Result in thread 0.
template <int NT>
__device__ __forceinline__ double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = (l < NT / 32) ? sh[l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_down_sync(0xffffffffu, r, o));
    }
    __syncthreads();
    return r;
}

// block_max and block_sum of two values at once, with the same orders (so
// the same bits) and one barrier pair instead of two.  Results in thread 0.
template <int NT>
__device__ __forceinline__ void block_max_sum(double& vmax_, double& vsum, double* sh /* >= 2 NT/32 */) {
    for (int o = 16; o > 0; o >>= 1) {
        vmax_ = fmax(vmax_, __shfl_down_sync(0xffffffffu, vmax_, o));
        vsum += __shfl_down_sync(0xffffffffu, vsum, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) { sh[w] = vmax_; sh[NT / 32 + w] = vsum; }
    __syncthreads();
    if (w == 0) {
        double m = (l < NT / 32) ? sh[l] : 0.0, r = (l < NT / 32) ? sh[NT / 32 + l] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
            r += __shfl_down_sync(0xffffffffu, r, o);
        }
        vmax_ = m;
        vsum = r;
    }
    __syncthreads();
}

// Grid-wide barrier for kernels launched cooperatively (all blocks resident).
// Sense is a generation counter.  The wait is bounded: after max_spins polls the
// block records an error in *err and leaves; callers test the return value and
// stop their loop, so a failed barrier ends the kernel instead of hanging it.
struct GridBarrier {
    unsigned int* count;   // zero-initialised
    unsigned int* gen;     // any start value
    int* err;              // zero-initialised; set to 1 on timeout
};

__device__ __forceinline__ bool grid_sync(const GridBarrier& b, unsigned nblocks) {
    __syncthreads();
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        volatile unsigned int* vgen = b.gen;
        unsigned int g = *vgen;
        __threadfence();
        unsigned int arrived = atomicAdd(b.count, 1u);
        int ok = 1;
        if (arrived == nblocks - 1) {
            atomicExch(b.count, 0u);
            __threadfence();
            atomicAdd(b.gen, 1u);
        } else {
            long long spins = 0;
            while (*vgen == g) {
                if (*(volatile int*)b.err) { ok = 0; break; }
                if (++spins > (1ll << 24)) { atomicExch(b.err, 1); ok = 0; break; }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace ccb
