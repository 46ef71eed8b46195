// Batched ensemble of independent 2D resistive-MHD instances (templated on T).
//
// Every instance keeps the single-grid device layout (three rotating pitched
// state buffers of 8 fields, a pitched phi) inside one pool; a device table of
// BatchInst records holds its constants and pointers.  All instances step in
// lockstep (the rotation index is shared) but each has its own dt, t, t_end
// and active flag, so an instance that reaches t_end simply carries its state.
//
// Work-lists are flat arrays of tiles {instance, (ty << 16) | tx}, instance by
// instance:
//   stage tiles   TX x TY cells, one per m2_stage_tile call (the single-grid
//                 stage body); the persistent stage kernel gives each CTA a
//                 contiguous run of the list, so consecutive tiles mostly share
//                 an instance and its record stays in shared memory;
//   reduce tiles  RTX x RTY cells, one warp per tile (the partial of a one-thread-per-cell block reduction), one partial (max CFL
//                 speed, density sum) per tile; an instance's partials are a
//                 contiguous range reduced in a fixed order, so every per-
//                 instance reduction is deterministic and independent of the
//                 other instances in the batch.
#pragma once
#include "mhd2d_kernels.cuh"

namespace ccb {

constexpr int RTX = 32, RTY = 8, RNT = RTX * RTY;   // reduction tile

// Constants and pointers of one instance (device table entry).
template <class T> struct BatchInst {
    M2Const<T> c;
    Fields<T> buf[3];
    T* phi;               // pitched gravitational potential (stage gravity source)
    // direct Poisson solve in the state precision T (FP64 instances: the
    // bitwise-reproducible path; FP32 instances: FP32 bases, factors and
    // work array): x transform by a dense orthonormal basis, then one
    // tridiagonal (or cyclic) solve per x wavenumber along y
    const T* tx;          // nx*nx: row k = k-th basis vector of the x second difference
    const T* txt;         // its transpose
    const T* lamx;        // nx eigenvalues of the x second difference (1/dx^2 units included)
    T* ah;                // ny*nx: transformed rhs, then transformed phi (in place)
    // factors of the y systems, [j*nx + k] (set up once per grid shape):
    const T* ycp;         // Thomas cp_j
    const T* yinv;        // 1 / m_j
    const T* yz;          // cyclic correction vector (periodic y only)
    const T* yfden;       // nx: 1 / (1 + v.z) (periodic y only)
    double fourpiG;
    double ay;            // 1/dy^2
    double dy2;           // dy^2
    T* rec[6];            // stage record (pre-floor update), written by the REC stage variant
};

// Per-instance reduction bookkeeping (precision independent).
struct BatchRed {
    int base, count;      // range of reduce tiles
    double ncell;
    DtSpec dts;
};

__device__ __forceinline__ void unpack_tile(int2 w, int& tx, int& ty) { tx = w.y & 0xffff; ty = w.y >> 16; }

// Copy one instance record into shared memory (all threads call; ends with a barrier).
template <class T>
__device__ __forceinline__ void load_inst(BatchInst<T>* dst, const BatchInst<T>* __restrict__ src) {
    constexpr int NW = (int)(sizeof(BatchInst<T>) / sizeof(int));
    static_assert(sizeof(BatchInst<T>) % sizeof(int) == 0, "record size");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(dst);
    for (int k = threadIdx.x; k < NW; k += blockDim.x) d[k] = s[k];
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Persistent stage kernel: a contiguous run of the stage work-list per CTA.
// src/dst index the instance's rotating buffers; gravity from phi (GRAV_PHI)
// or none.
// ---------------------------------------------------------------------------
template <class T, int TX, int TY, int NT, int MINB, bool SPLIT, bool DEFER, int GMODE, bool REC = false>
__global__ void __launch_bounds__(NT, MINB)
m2b_stage_kernel(const BatchInst<T>* __restrict__ inst, const int2* __restrict__ work, int nwork, int src, int dst,
                 const double* __restrict__ dt, const int* __restrict__ active) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) BatchInst<T> s_inst;
    T* sm = reinterpret_cast<T*>(smem_raw);
    const int per = (nwork + (int)gridDim.x - 1) / (int)gridDim.x;
    const int w0 = (int)blockIdx.x * per;
    const int w1 = min(nwork, w0 + per);
    int cur = -1;
    for (int w = w0; w < w1; ++w) {
        const int2 it = work[w];
        if (active[it.x] == 0) continue;            // uniform over the CTA
        if (it.x != cur) {
            __syncthreads();                        // previous tile done with s_inst
            load_inst(&s_inst, inst + it.x);
            cur = it.x;
        }
        int tx, ty;
        unpack_tile(it, tx, ty);
        m2_stage_tile<T, TX, TY, DEFER, GMODE, REC, NT, SPLIT>(s_inst.c, s_inst.buf[src], s_inst.buf[dst], s_inst.phi,
                                                        nullptr, (T)dt[it.x], tx * TX, ty * TY, sm, s_inst.rec);
        __syncthreads();                            // shared tile buffers reused by the next tile
    }
}

// ---------------------------------------------------------------------------
// Reduce tiles are worked by one warp each (RNT/32 tiles per CTA, no block
// barriers): lane = column, the RTY rows in turn.  The partials are the same
// doubles as block_max_sum / block_sum over the tile with one thread per cell
// (warp = row): each row's values go through that warp shuffle tree, the row
// results are placed in lanes 0..RTY-1 (the other lanes 0) and go through the
// same second-level tree.
// ---------------------------------------------------------------------------
constexpr int RWPB = RNT / 32;   // reduce tiles per CTA
static_assert(RTX == 32 && RTY <= 32, "a reduce-tile row is one warp");

__device__ __forceinline__ void rtile_tree(double& m, double& s) {
    for (int o = 16; o > 0; o >>= 1) {
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
        s += __shfl_down_sync(0xffffffffu, s, o);
    }
}

// fold row r's (max, sum) into the lane-r slot of the second level
__device__ __forceinline__ void rtile_row(int r, double m, double s, double& rm, double& rs) {
    rtile_tree(m, s);
    m = __shfl_sync(0xffffffffu, m, 0);
    s = __shfl_sync(0xffffffffu, s, 0);
    if ((threadIdx.x & 31) == r) { rm = m; rs = s; }
}

// ---------------------------------------------------------------------------
// RK average over reduce tiles: U^{n+1} = average(U^n, Joule(S2)) with floors,
// plus the per-tile CFL-speed max and density sum of U^{n+1}.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(RNT)
m2b_average_kernel(const BatchInst<T>* __restrict__ inst, const int2* __restrict__ rwork, int nrwork, int a, int d,
                   int b, const double* __restrict__ dt, const int* __restrict__ active,
                   double* __restrict__ spd_part, double* __restrict__ rho_part) {
    const int lane = threadIdx.x & 31;
    for (int w = blockIdx.x * RWPB + (threadIdx.x >> 5); w < nrwork; w += gridDim.x * RWPB) {
        const int2 it = rwork[w];
        const BatchInst<T>& I = inst[it.x];
        int tx, ty;
        unpack_tile(it, tx, ty);
        const int i = tx * RTX + lane;
        const bool act = active[it.x] != 0;
        const T dtv = (T)dt[it.x];
        double rm = 0.0, rs = 0.0;
        for (int r = 0; r < RTY; r++) {
            const int j = ty * RTY + r;
            double smax = 0.0, rsum = 0.0;
            if (i < I.c.nx && j < I.c.ny) {
                const double v = average_cell(I.c, I.buf[a], I.buf[d], I.buf[b], dtv, act, i, j, rsum);
                if (v > smax) smax = v;
            }
            rtile_row(r, smax, rsum, rm, rs);
        }
        rtile_tree(rm, rs);
        if (lane == 0) { spd_part[w] = rm; rho_part[w] = rs; }
    }
}

// CFL speed max and density sum per reduce tile of buffer src.
template <class T>
__global__ void __launch_bounds__(RNT)
m2b_speed_kernel(const BatchInst<T>* __restrict__ inst, const int2* __restrict__ rwork, int nrwork, int src,
                 double* __restrict__ spd_part, double* __restrict__ rho_part) {
    const int lane = threadIdx.x & 31;
    for (int w = blockIdx.x * RWPB + (threadIdx.x >> 5); w < nrwork; w += gridDim.x * RWPB) {
        const int2 it = rwork[w];
        const BatchInst<T>& I = inst[it.x];
        int tx, ty;
        unpack_tile(it, tx, ty);
        const int i = tx * RTX + lane;
        double rm = 0.0, rs = 0.0;
        for (int r = 0; r < RTY; r++) {
            const int j = ty * RTY + r;
            double smax = 0.0, rsum = 0.0;
            if (i < I.c.nx && j < I.c.ny) {
                const double v = speed_cell(I.c, I.buf[src], i, j);
                if (v > smax) smax = v;
                rsum = (double)I.buf[src].rho[(size_t)j * I.c.pitch + i];
            }
            rtile_row(r, smax, rsum, rm, rs);
        }
        rtile_tree(rm, rs);
        if (lane == 0) { spd_part[w] = rm; rho_part[w] = rs; }
    }
}

// Density sum per reduce tile of buffer src (the Poisson mean of stage 1's output).
template <class T>
__global__ void __launch_bounds__(RNT)
m2b_rho_sum_kernel(const BatchInst<T>* __restrict__ inst, const int2* __restrict__ rwork, int nrwork, int src,
                   const int* __restrict__ active, double* __restrict__ rho_part) {
    const int lane = threadIdx.x & 31;
    for (int w = blockIdx.x * RWPB + (threadIdx.x >> 5); w < nrwork; w += gridDim.x * RWPB) {
        const int2 it = rwork[w];
        if (active[it.x] == 0) continue;   // uniform over the warp
        const BatchInst<T>& I = inst[it.x];
        int tx, ty;
        unpack_tile(it, tx, ty);
        const int i = tx * RTX + lane;
        double rm = 0.0, rs = 0.0;
        for (int r = 0; r < RTY; r++) {
            const int j = ty * RTY + r;
            const double rsum = (i < I.c.nx && j < I.c.ny) ? (double)I.buf[src].rho[(size_t)j * I.c.pitch + i] : 0.0;
            rtile_row(r, 0.0, rsum, rm, rs);
        }
        rtile_tree(rm, rs);
        if (lane == 0) rho_part[w] = rs;
    }
}

}  // namespace ccb
