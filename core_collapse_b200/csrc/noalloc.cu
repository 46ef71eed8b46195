// cc_mhd2d_gravity_fft_noalloc: the spectral self-gravity solve of
// cc_mhd2d_compute_gravity (FFT path, FP64) for callers that cannot allocate
// device memory.  All scratch -- the complex work array, the potential, the
// density partial sums and the four twiddle tables -- lives in one file-scope
// device array of fixed size, so the call makes no cudaMalloc/cudaFree and
// calls no allocating library routine.  The caller passes device pointers for
// the input density and the output acceleration.
//
// Built with -fmad=false like the other FP64 kernels.
#include <mutex>

#include "../../include/cc_step.h"
#include "mhd2d_launch.h"

namespace ccb {
namespace {

// Scratch layout in doubles; every region starts on a 256-byte boundary.
constexpr size_t NA_MAX_CELLS = CC_NOALLOC_MAX_CELLS;
constexpr size_t NA_MAX_SIDE = CC_NOALLOC_MAX_SIDE;
constexpr size_t NA_A = 0;                                   // complex work array: 2 * max cells
constexpr size_t NA_PHI = NA_A + 2 * NA_MAX_CELLS;           // potential: max cells
constexpr size_t NA_PART = NA_PHI + NA_MAX_CELLS;            // RED_BLOCKS density partial sums
constexpr size_t NA_TW = NA_PART + 320;                      // 4 twiddle tables, 2 * max side each
constexpr size_t NA_TWSZ = 2 * NA_MAX_SIDE;
constexpr size_t NA_TOTAL = NA_TW + 4 * NA_TWSZ;
static_assert(RED_BLOCKS <= 320, "partial-sum region too small");
static_assert(NA_PHI % 32 == 0 && NA_PART % 32 == 0 && NA_TW % 32 == 0 && NA_TWSZ % 32 == 0, "alignment");

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) double cc_noalloc_scratch[NA_TOTAL];

// Twiddles of each radix-2 pass of an n-point transform, one thread per pass,
// by the recurrence w_{j+1} = w_j * wlen of the reference FFT
// (navier_stokes_2d_hllc_poisson.cpp:160-171); pass of half-length h at [h-1, 2h-1).
// wlen comes from the device's cos/sin, where the handle path builds its table
// on the host with the C library's: the two can differ in the last bit of wlen,
// so this solve agrees with cc_mhd2d_compute_gravity to about 1e-13 relative,
// not bit for bit.
__global__ void na_twiddle_kernel(Cplx<double>* tw, int n, int inverse) {
    const int pass = blockIdx.x * blockDim.x + threadIdx.x;
    if (pass >= 31) return;
    const int len = 2 << pass;
    if (len > n) return;
    const double ang = 2.0 * M_PI / len * (inverse ? +1.0 : -1.0);
    const double wr = cos(ang), wi = sin(ang);
    double cr = 1.0, ci = 0.0;
    const int h = len / 2;
    for (int j = 0; j < h; j++) {
        tw[h - 1 + j].re = cr;
        tw[h - 1 + j].im = ci;
        const double nr = cr * wr - ci * wi, ni = cr * wi + ci * wr;
        cr = nr;
        ci = ni;
    }
}

struct DeviceScratch {
    bool ready = false;
    double* base = nullptr;
};
std::mutex g_mutex;
DeviceScratch g_devices[128];

// First call on a device (that device current): resolve the array's device
// address -- in host code its name is only a host-side stand-in -- and raise
// the shared-memory limits of the FFT kernels to the largest allowed line.
int device_scratch(double** base) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return CC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    DeviceScratch& d = g_devices[dev];
    if (!d.ready) {
        void* ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, cc_noalloc_scratch) != cudaSuccess || ptr == nullptr) return CC_ERR_CUDA;
        if (M2Launch<double>::prepare((int)NA_MAX_SIDE, (int)NA_MAX_SIDE) != cudaSuccess) return CC_ERR_CUDA;
        d.base = static_cast<double*>(ptr);
        d.ready = true;
    }
    *base = d.base;
    return CC_OK;
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }
int log2i(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }

}  // namespace
}  // namespace ccb

using namespace ccb;

extern "C" int cc_mhd2d_gravity_fft_noalloc(const cc_mhd2d_params* p, const double* rho, double* gx, double* gy,
                                            void* stream) {
    if (!p || !rho || !gx || !gy) return CC_ERR_ARG;
    const int nx = p->Nx, ny = p->Ny;
    if (p->precision != CC_FP64 || p->poisson_kind != CC_POISSON_FFT || !p->periodic_x || !p->periodic_y)
        return CC_ERR_UNSUPPORTED;
    if (!pow2(nx) || !pow2(ny) || nx < 4 || ny < 4) return CC_ERR_UNSUPPORTED;
    if ((size_t)nx > NA_MAX_SIDE || (size_t)ny > NA_MAX_SIDE || (size_t)nx * (size_t)ny > NA_MAX_CELLS)
        return CC_ERR_TOO_LARGE;
    if (!(p->x1 > p->x0) || !(p->y1 > p->y0)) return CC_ERR_ARG;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const size_t nbytes = sizeof(double) * (size_t)nx * ny;
    if (!p->gravity_on) {
        if (cudaMemsetAsync(gx, 0, nbytes, s) != cudaSuccess || cudaMemsetAsync(gy, 0, nbytes, s) != cudaSuccess)
            return CC_ERR_CUDA;
        return CC_OK;
    }
    double* base = nullptr;
    if (int r = device_scratch(&base)) return r;
    Cplx<double>* A = reinterpret_cast<Cplx<double>*>(base + NA_A);
    double* phi = base + NA_PHI;
    double* part = base + NA_PART;
    Cplx<double>* tw[4];
    for (int k = 0; k < 4; k++) tw[k] = reinterpret_cast<Cplx<double>*>(base + NA_TW + k * NA_TWSZ);

    const double dx = (p->x1 - p->x0) / nx, dy = (p->y1 - p->y0) / ny;
    M2Const<double> c{};
    c.nx = nx; c.ny = ny; c.pitch = nx;   // contiguous caller arrays
    const AxisMap ax{nx, 1}, ay{ny, 1};
    const int lx = log2i(nx), ly = log2i(ny);

    if (M2Launch<double>::rho_sum(c, rho, part, s) != cudaSuccess) return CC_ERR_CUDA;
    na_twiddle_kernel<<<1, 32, 0, s>>>(tw[0], nx, 0);
    na_twiddle_kernel<<<1, 32, 0, s>>>(tw[1], nx, 1);
    na_twiddle_kernel<<<1, 32, 0, s>>>(tw[2], ny, 0);
    na_twiddle_kernel<<<1, 32, 0, s>>>(tw[3], ny, 1);
    if (cudaGetLastError() != cudaSuccess) return CC_ERR_CUDA;
    if (M2Launch<double>::fft_solve(rho, nx, part, nx, ny, lx, ly, tw[0], tw[1], tw[2], tw[3], p->x1 - p->x0,
                                    p->y1 - p->y0, p->G, A, phi, nullptr, s) != cudaSuccess)
        return CC_ERR_CUDA;
    if (M2Launch<double>::gravity_from_phi(phi, nx, ny, nx, ax, ay, 2.0 * dx, 2.0 * dy, gx, gy, s) != cudaSuccess)
        return CC_ERR_CUDA;
    return CC_OK;
}
