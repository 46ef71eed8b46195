// Reverse of the red-black SOR Poisson solve (M2:178-237 in the red-black
// order of sor_rb_kernel), for the discrete adjoint.
//
// With a fixed number of sweeps K (or the recorded count of a tolerance-
// stopped solve) the solve is a linear map of its right-hand side: from
// phi = 0, each sweep is a red half-sweep, a black half-sweep, and the
// removal of the mean,
//   phi_c <- (1 - omega) phi_c + omega / den (sum_n w_n phi_n - rhs_c)
// for the cells c of one colour, n the four neighbours under the axis maps
// (a clamped neighbour may be c itself), w_n = 1/dx^2 or 1/dy^2.  Its adjoint
// runs the sweeps backwards: mean removal (symmetric), black half-sweep
// transposed, red half-sweep transposed.  A transposed half-sweep scales the
// adjoint of each updated cell by (1 - omega) + omega w_self / den, adds to
// each other cell the adjoint of its updated neighbours times omega w / den
// (the stencil is symmetric: a cell reads its neighbour exactly when the
// neighbour reads it), and adds -omega / den times the updated cell's adjoint
// to the adjoint of the right-hand side.  One kernel per half-sweep over all
// cells, from one adjoint buffer into the other; the mean removal rides on the
// black kernel, which reads its input minus the mean of the previous red
// kernel's output (partial sums from that kernel).  No grid barrier.
#pragma once
#include "cc_device.cuh"

namespace ccb {

constexpr int ASOR_NT = 256;
constexpr int ASOR_BLOCKS = 296;

struct SorAdjArgs {
    int nx, ny;
    AxisMap ax, ay;
    double idx2, idy2, denom, omega;
    double* rhat;        // adjoint of the right-hand side (accumulated), nx*ny
    double* part;        // ASOR_BLOCKS partial sums
};

// rhs = 4 pi G (rho - mean) of a pitched density with a device mean (M2:187-194)
template <class T>
__global__ void adj_sor_rhs_kernel(const T* __restrict__ rho, int nx, int ny, int P, const double* __restrict__ mean,
                                   double fourpiG, double* __restrict__ rhs, const int* __restrict__ active) {
    if (active && *active == 0) return;
    const double m = *mean;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nx * ny; k += gridDim.x * blockDim.x)
        rhs[k] = fourpiG * ((double)rho[(size_t)(k / nx) * P + (k % nx)] - m);
}

// mu = the pitched adjoint of phi (T) as a contiguous FP64 field; partial sums
// for the first mean removal; rhat zeroed
template <class T>
__global__ void __launch_bounds__(ASOR_NT)
adj_sor_start_kernel(SorAdjArgs a, const T* __restrict__ lphi, int P, double* __restrict__ mu) {
    __shared__ double sh[ASOR_NT / 32];
    double s = 0.0;
    for (int k = blockIdx.x * ASOR_NT + threadIdx.x; k < a.nx * a.ny; k += gridDim.x * ASOR_NT) {
        const double v = (double)lphi[(size_t)(k / a.nx) * P + (k % a.nx)];
        mu[k] = v;
        a.rhat[k] = 0.0;
        s += v;
    }
    s = block_sum<ASOR_NT>(s, sh);
    if (threadIdx.x == 0) a.part[blockIdx.x] = s;
}

// one transposed half-sweep of colour COLOR ((i + j) & 1 == COLOR updated);
// MEAN: read mu_in minus the mean of the partial sums; SUMS: partial sums of
// mu_out.  A block works whole rows (coalesced, no index division), the
// updated cells of a row and then the others (no divergence between them).
template <int COLOR, bool MEAN, bool SUMS>
__global__ void __launch_bounds__(ASOR_NT)
adj_sor_half_kernel(SorAdjArgs a, const double* __restrict__ mu_in, double* __restrict__ mu_out) {
    __shared__ double sh[ASOR_NT / 32];
    __shared__ double s_m;
    double m = 0.0;
    if constexpr (MEAN) {
        if (threadIdx.x < 32) {   // one warp sums the partials (fixed order)
            double t = 0.0;
            for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) t += a.part[b];
            for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
            if (threadIdx.x == 0) s_m = t / ((double)a.nx * (double)a.ny);
        }
        __syncthreads();
        m = s_m;
        __syncthreads();   // every block reads part before any block writes it (SUMS is off here)
    }
    const double k1 = a.omega / a.denom;
    const int nh = (a.nx + 1) / 2;
    double s = 0.0;
    for (int j = blockIdx.x; j < a.ny; j += gridDim.x) {
        const int jN = a.ay.cell(j + 1), jS = a.ay.cell(j - 1);
        const double* rowC = mu_in + (size_t)j * a.nx;
        const double* rowN = mu_in + (size_t)jN * a.nx;
        const double* rowS = mu_in + (size_t)jS * a.nx;
        double* out = mu_out + (size_t)j * a.nx;
        double* rh = a.rhat + (size_t)j * a.nx;
        const double yself = (jN == j ? a.idy2 : 0.0) + (jS == j ? a.idy2 : 0.0);
        // updated cells: (1 - omega + omega w_self / den) mu, and -omega/den mu into rhat
        for (int t = threadIdx.x; t < nh; t += ASOR_NT) {
            const int i = 2 * t + ((COLOR + j) & 1);
            if (i >= a.nx) continue;
            const int iE = a.ax.cell(i + 1), iW = a.ax.cell(i - 1);
            const double self = yself + (iE == i ? a.idx2 : 0.0) + (iW == i ? a.idx2 : 0.0);
            const double mq = rowC[i] - m;
            const double v = (1.0 - a.omega) * mq + k1 * self * mq;
            rh[i] -= k1 * mq;
            out[i] = v;
            s += v;
        }
        // the other cells gather the updated neighbours that read them
        for (int t = threadIdx.x; t < nh; t += ASOR_NT) {
            const int i = 2 * t + ((COLOR + j + 1) & 1);
            if (i >= a.nx) continue;
            const int iE = a.ax.cell(i + 1), iW = a.ax.cell(i - 1);
            double acc = 0.0;
            if (iE != i) acc += a.idx2 * (rowC[iE] - m);
            if (iW != i) acc += a.idx2 * (rowC[iW] - m);
            if (jN != j) acc += a.idy2 * (rowN[i] - m);
            if (jS != j) acc += a.idy2 * (rowS[i] - m);
            const double v = (rowC[i] - m) + k1 * acc;
            out[i] = v;
            s += v;
        }
    }
    if constexpr (SUMS) {
        s = block_sum<ASOR_NT>(s, sh);
        if (threadIdx.x == 0) a.part[blockIdx.x] = s;
    }
}

// partial sums of rhat (for its mean); NT = ASOR_NT
template <int NT>
__global__ void __launch_bounds__(NT) adj_sor_rhat_sum_kernel(SorAdjArgs a) {
    __shared__ double sh[NT / 32];
    double s = 0.0;
    for (int k = blockIdx.x * NT + threadIdx.x; k < a.nx * a.ny; k += gridDim.x * NT) s += a.rhat[k];
    s = block_sum<NT>(s, sh);
    if (threadIdx.x == 0) a.part[blockIdx.x] = s;
}

// rhs = 4 pi G (rho - mean(rho)) in reverse: lrho += 4 pi G (rhat - mean(rhat))
template <class T>
__global__ void __launch_bounds__(ASOR_NT)
adj_sor_finish_kernel(SorAdjArgs a, double fourpiG, T* __restrict__ lrho, int P) {
    __shared__ double s_m;
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) t += a.part[b];
        s_m = t / ((double)a.nx * (double)a.ny);
    }
    __syncthreads();
    const double m = s_m;
    for (int k = blockIdx.x * ASOR_NT + threadIdx.x; k < a.nx * a.ny; k += gridDim.x * ASOR_NT) {
        const size_t q = (size_t)(k / a.nx) * P + (k % a.nx);
        lrho[q] += (T)(fourpiG * (a.rhat[k] - m));
    }
}

}  // namespace ccb
