// Tensor-core (tcgen05) basis transforms of the batched direct Poisson solve
// for FP32 instances: the two dense products of dp_gemm_kernel,
//   MODE 0:  ah  = (4 pi G (rho - mean)) * Tx^T      (ny x nx) * (nx x nx)
//   MODE 1:  phi = ah * Tx
// on 128 x 128 output tiles, FP32 accuracy from three TF32 products: every
// operand is split x = hi + lo with hi = x rounded to TF32 (11 significant
// bits, round half away from zero), lo = x - hi (exact in FP32, |lo| <=
// 2^-12 |x|) also rounded to TF32 (the tensor core would otherwise truncate
// it), and C = A_hi B_hi + A_hi B_lo + A_lo B_hi with FP32 accumulation in
// tensor memory: about 2^-23 relative per product (the dropped A_lo B_lo term
// is 2^-24).
//
// Per CTA (256 threads, one output tile):
//   * warp 0 allocates 128 TMEM columns (the 128 x 128 FP32 accumulator);
//   * K runs in chunks of 16: all threads load the A and B chunks from global
//     memory (B = rows of Tx or Tx^T, i.e. both operands K-major), split them
//     and store hi and lo parts to shared memory in the canonical K-major
//     no-swizzle layout -- 16-byte core-matrix rows, unit (kc, row) at byte
//     (kc * 128 + row) * 16, so 8-row groups are 128 B apart (SBO) and the two
//     16-byte K halves of one MMA are 2048 B apart (LBO); the global loads of
//     chunk c+2 are issued into registers right after chunk c is stored, so
//     their latency overlaps two iterations (barriers and MMAs);
//   * one thread issues the 2 K-steps x 3 products of the chunk
//     (tcgen05.mma.cta_group::1.kind::tf32, M = N = 128, K = 8) and commits
//     them to the chunk's mbarrier; two shared-memory stages, so the stores of
//     chunk c+1 overlap the MMAs of chunk c;
//   * epilogue: each warp reads 32 accumulator lanes (rows) x 64 columns with
//     tcgen05.ld and stores them (float4) to ah or phi.
// Every mbarrier wait is bounded; on a timeout the kernel sets bit 0 of *err,
// waits (bounded) for its own MMAs, frees its TMEM and returns.  If that last
// wait gives up too, MMAs may still be writing the TMEM it frees: the kernel
// then also sets bit 1, and the handle refuses all further work.
#pragma once
#include <cstdint>

#include "batch_kernels.cuh"

namespace ccb {

constexpr int TCM = 128, TCN = 128, TCK = 16, TCNT = 256;
constexpr int TCU = TCM * (TCK / 4) / TCNT;              // 16-byte units per thread and operand per chunk
constexpr int TC_PART = TCM * TCK * 4;                   // bytes of one operand part (A or B, hi or lo)
constexpr int TC_STAGE = 4 * TC_PART;                    // A hi, A lo, B hi, B lo
constexpr int TC_SMEM = 2 * TC_STAGE + 64;               // two stages, two mbarriers, the TMEM address
                                                         // (64 KB: three CTAs per SM, 384 TMEM columns)
constexpr unsigned TC_WAIT_POLLS = 1u << 24;             // x >= 64 ns sleep: > 1 s before giving up

// instruction descriptor: D FP32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2),
// both K-major (bits 15, 16 = 0), N >> 3 at bit 17, M >> 4 at bit 24
constexpr uint32_t TC_IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TCN >> 3) << 17) |
                              ((uint32_t)(TCM >> 4) << 24);

__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor, no swizzle: start >> 4 (bits 0-13),
// leading (K) byte offset >> 4 (16-29), stride (8-row group) byte offset >> 4
// (32-45), descriptor version 1 (bits 46-47), base offset 0, layout 0
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(TC_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void tc_mbar_init(uint32_t mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(mbar) : "memory");
}

// true once phase `parity` of the mbarrier has completed; false after the poll limit
__device__ __forceinline__ bool tc_mbar_wait(uint32_t mbar, uint32_t parity) {
    for (unsigned it = 0; it < TC_WAIT_POLLS; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (done) return true;
        __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 32 consecutive FP32 columns of the accumulator into v
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// nearest TF32 value (11 significant bits; half-way rounds away from zero)
__device__ __forceinline__ float tc_tf32(float x) {
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}
__device__ __forceinline__ float4 tc_tf32(float4 v) {
    return make_float4(tc_tf32(v.x), tc_tf32(v.y), tc_tf32(v.z), tc_tf32(v.w));
}
__device__ __forceinline__ float4 tc_lo(float4 v, float4 h) {
    return tc_tf32(make_float4(v.x - h.x, v.y - h.y, v.z - h.z, v.w - h.w));
}

// gwork items {instance, (tm << 16) | tn} of 128 x 128 tiles; instances with
// nx a multiple of 4 (16-byte rows).
template <int MODE>
__global__ void __launch_bounds__(TCNT, 3)
dp_gemm_tc_kernel(const BatchInst<float>* __restrict__ inst, const int2* __restrict__ gwork, int src,
                  const double* __restrict__ rho_mean, const int* __restrict__ active, int* __restrict__ err) {
    const int2 it = gwork[blockIdx.x];
    if (active[it.x] == 0) return;   // uniform over the CTA
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    const BatchInst<float>& I = inst[it.x];
    const int nx = I.c.nx, ny = I.c.ny, P = I.c.pitch;
    const int m0 = (it.y >> 16) * TCM, n0 = (it.y & 0xffff) * TCN;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint64_t* mbar = reinterpret_cast<uint64_t*>(tc_smem + 2 * TC_STAGE);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(tc_smem + 2 * TC_STAGE + 16);
    volatile int* sok = reinterpret_cast<volatile int*>(tc_smem + 2 * TC_STAGE + 32);   // wait outcome, broadcast
    const uint32_t mb0 = tc_smem_addr(&mbar[0]), mb1 = tc_smem_addr(&mbar[1]);

    if (tid == 0) {
        tc_mbar_init(mb0);
        tc_mbar_init(mb1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(tslot)),
                     "r"(TCN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    const float* __restrict__ Bsrc = (MODE == 0) ? I.tx : I.txt;   // row n = K-major row of B
    const float mean = (MODE == 0) ? (float)rho_mean[it.x] : 0.0f;
    const float fpg = (float)I.fourpiG;
    const int nk = (nx + TCK - 1) / TCK;
    bool ok = true;
    int issued = 0;   // chunks whose MMAs were committed

    // operands of two chunks in registers (slot = chunk parity): the loads of
    // chunk c+2 are issued as soon as chunk c is in shared memory, two
    // iterations ahead of their use
    float4 ra[2][TCU], rb[2][TCU];
    auto gload = [&](int c, float4* xa, float4* xb) {
        const int k0 = c * TCK;
#pragma unroll
        for (int i = 0; i < TCU; i++) {
            const int u = tid + i * TCNT, kc = u >> 7, row = u & 127;
            const int gk = k0 + 4 * kc, gm = m0 + row, gn = n0 + row;
            xa[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            xb[i] = xa[i];
            if (gm < ny && gk < nx) {
                if (MODE == 0) xa[i] = *reinterpret_cast<const float4*>(I.buf[src].rho + (size_t)gm * P + gk);
                else xa[i] = *reinterpret_cast<const float4*>(I.ah + (size_t)gm * nx + gk);
            }
            if (gn < nx && gk < nx) xb[i] = *reinterpret_cast<const float4*>(Bsrc + (size_t)gn * nx + gk);
        }
    };
    // one K chunk: wait until its stage is free, split and store, prefetch
    // chunk c+2, hand the stage to the tensor core; false after a timed-out wait
    auto chunk = [&](int c, float4* xa, float4* xb) -> bool {
        const int s = c & 1;
        unsigned char* stage = tc_smem + s * TC_STAGE;
        if (c >= 2) {   // the MMAs of chunk c-2 read this stage: thread 0 waits, the CTA follows
            if (tid == 0) *sok = tc_mbar_wait(s ? mb1 : mb0, (uint32_t)(((c - 2) >> 1) & 1)) ? 1 : 0;
            __syncthreads();
            if (*sok == 0) return false;   // uniform
        }
        // 128 rows x TCK/4 sixteen-byte units per operand; unit u -> (kc = u / 128, row = u % 128)
#pragma unroll
        for (int i = 0; i < TCU; i++) {
            const int u = tid + i * TCNT, kc = u >> 7, row = u & 127;
            const int gk = c * TCK + 4 * kc, gm = m0 + row;
            float4 a = xa[i];
            if (MODE == 0) {   // 4 pi G (rho - mean) inside the instance, 0 in the padding
                const bool in = gm < ny && gk < nx;
                a = in ? make_float4(fpg * (a.x - mean), fpg * (a.y - mean), fpg * (a.z - mean), fpg * (a.w - mean))
                       : make_float4(0.f, 0.f, 0.f, 0.f);
            }
            const float4 b = xb[i];
            const float4 ah = tc_tf32(a), bh = tc_tf32(b);
            const int off = (kc * 128 + row) * 16;
            *reinterpret_cast<float4*>(stage + off) = ah;
            *reinterpret_cast<float4*>(stage + TC_PART + off) = tc_lo(a, ah);
            *reinterpret_cast<float4*>(stage + 2 * TC_PART + off) = bh;
            *reinterpret_cast<float4*>(stage + 3 * TC_PART + off) = tc_lo(b, bh);
        }
        if (c + 2 < nk) gload(c + 2, xa, xb);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const uint32_t base = tc_smem_addr(stage);
#pragma unroll
            for (int ks = 0; ks < TCK / 8; ks++) {
                const uint32_t kofs = (uint32_t)ks * 2 * 2048;   // two 16-byte K units per MMA
                const uint64_t dah = tc_desc(base + kofs, 2048, 128);
                const uint64_t dal = tc_desc(base + TC_PART + kofs, 2048, 128);
                const uint64_t dbh = tc_desc(base + 2 * TC_PART + kofs, 2048, 128);
                const uint64_t dbl = tc_desc(base + 3 * TC_PART + kofs, 2048, 128);
                tc_mma(tmem, dah, dbh, (c > 0 || ks > 0) ? 1u : 0u);
                tc_mma(tmem, dah, dbl, 1u);
                tc_mma(tmem, dal, dbh, 1u);
            }
            tc_commit(s ? mb1 : mb0);
        }
        issued = c + 1;
        return true;
    };
    gload(0, ra[0], rb[0]);
    if (nk > 1) gload(1, ra[1], rb[1]);
    for (int c = 0; c < nk; c += 2) {
        if (!chunk(c, ra[0], rb[0])) { ok = false; break; }
        if (c + 1 < nk && !chunk(c + 1, ra[1], rb[1])) { ok = false; break; }
    }
    // wait for the last committed chunk (a commit tracks all earlier MMAs of the thread)
    if (tid == 0) {
        bool done = true;
        if (issued > 0) {
            const int c = issued - 1;
            done = tc_mbar_wait((c & 1) ? mb1 : mb0, (uint32_t)((c >> 1) & 1));
        }
        if (!done) atomicOr(err, 3);   // the MMAs may outlive this CTA's TMEM
        *sok = (ok && done) ? 1 : 0;
    }
    __syncthreads();
    ok = *sok != 0;
    tc_fence_after();
    if (ok && issued == nk) {
        const int row = 32 * (warp & 3) + lane, h = warp >> 2;
        const int gm = m0 + row;
#pragma unroll
        for (int half = 0; half < 2; half++) {
            const int col = 64 * h + 32 * half;
            float v[32];
            tc_ld32(tmem + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)col, v);
            if (gm < ny) {
                float* dst = (MODE == 0) ? I.ah + (size_t)gm * nx : I.phi + (size_t)gm * P;
#pragma unroll
                for (int q = 0; q < 8; q++) {
                    const int gn = n0 + col + 4 * q;
                    if (gn < nx)
                        *reinterpret_cast<float4*>(dst + gn) = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
                }
            }
        }
    } else if (tid == 0) {
        atomicOr(err, 1);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCN));
    }
}

}  // namespace ccb
