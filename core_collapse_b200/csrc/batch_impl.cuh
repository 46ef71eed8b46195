// Definitions of BatchLaunch<T>; included once per precision TU.
//
// Stage tile candidates (TX, TY, threads, CTAs per SM the launch bounds ask
// for, split x/y slope buffers):
//   FP64: 32x8/256 (2), 16x16/256 (2)
//   FP32: 32x16/512 (2, split), 32x8/256 (4), 64x8/512 (2), 32x14/544 (2, split),
//         30x15/544 (2, one row per warp in every phase), 30x6/256 (4, the same)
// The autotuner of the batch handle times each on the actual work-list.
#pragma once
#include "batch_launch.h"

namespace ccb {

template <class T> struct BatchShapes;
template <> struct BatchShapes<double> {
    static constexpr int N = 2;
    template <int K> struct S;
};
template <> template <> struct BatchShapes<double>::S<0> {
    static constexpr int TX = 32, TY = 8, NT = 256, MINB = 2; static constexpr bool SPLIT = false;
};
template <> template <> struct BatchShapes<double>::S<1> {
    static constexpr int TX = 16, TY = 16, NT = 256, MINB = 2; static constexpr bool SPLIT = false;
};
template <> struct BatchShapes<float> {
    static constexpr int N = 6;
    template <int K> struct S;
};
template <> template <> struct BatchShapes<float>::S<0> {
    static constexpr int TX = 32, TY = 16, NT = 512, MINB = 2; static constexpr bool SPLIT = true;
};
template <> template <> struct BatchShapes<float>::S<1> {
    static constexpr int TX = 32, TY = 8, NT = 256, MINB = 4; static constexpr bool SPLIT = false;
};
template <> template <> struct BatchShapes<float>::S<2> {
    static constexpr int TX = 64, TY = 8, NT = 512, MINB = 2; static constexpr bool SPLIT = false;
};
template <> template <> struct BatchShapes<float>::S<3> {
    static constexpr int TX = 32, TY = 14, NT = 544, MINB = 2; static constexpr bool SPLIT = true;
};
template <> template <> struct BatchShapes<float>::S<4> {   // one row per warp in every phase (ROW32)
    static constexpr int TX = 30, TY = 15, NT = 544, MINB = 2; static constexpr bool SPLIT = false;
};
template <> template <> struct BatchShapes<float>::S<5> {   // the same on 8 warps, four CTAs per SM
    static constexpr int TX = 30, TY = 6, NT = 256, MINB = 4; static constexpr bool SPLIT = false;
};

namespace {

template <class T, int K> struct ShapeOps {
    using S = typename BatchShapes<T>::template S<K>;
    static constexpr size_t smem() { return StageGeomT<T, S::TX, S::TY, S::NT, S::SPLIT>::smem; }
    template <bool D, int G, bool R = false> static auto kern() {
        return m2b_stage_kernel<T, S::TX, S::TY, S::NT, S::MINB, S::SPLIT, D, G, R>;
    }
    static cudaError_t prepare_rec() {
        cudaError_t e;
        const int b = (int)smem();
        if ((e = cudaFuncSetAttribute(kern<false, GRAV_NONE, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
        if ((e = cudaFuncSetAttribute(kern<false, GRAV_PHI, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
        if ((e = cudaFuncSetAttribute(kern<true, GRAV_NONE, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
        return cudaFuncSetAttribute(kern<true, GRAV_PHI, true>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    }
    static cudaError_t stage_rec(int grid, const BatchInst<T>* inst, const int2* work, int nwork, int src, int dst,
                                 bool defer, bool grav, const double* dt, const int* active, cudaStream_t s) {
        const dim3 b(S::NT);
        if (defer && grav) kern<true, GRAV_PHI, true>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        else if (defer) kern<true, GRAV_NONE, true>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        else if (grav) kern<false, GRAV_PHI, true>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        else kern<false, GRAV_NONE, true>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        return cudaGetLastError();
    }
    static cudaError_t prepare() {
        cudaError_t e;
        const int b = (int)smem();
        if ((e = cudaFuncSetAttribute(kern<false, GRAV_NONE>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
        if ((e = cudaFuncSetAttribute(kern<false, GRAV_PHI>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
        if ((e = cudaFuncSetAttribute(kern<true, GRAV_NONE>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b))) return e;
        return cudaFuncSetAttribute(kern<true, GRAV_PHI>(), cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    }
    static cudaError_t resident(int* per_sm) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern<false, GRAV_PHI>(), S::NT, smem());
    }
    static cudaError_t stage(int grid, const BatchInst<T>* inst, const int2* work, int nwork, int src, int dst,
                             bool defer, bool grav, const double* dt, const int* active, cudaStream_t s) {
        const dim3 b(S::NT);
        if (defer && grav) kern<true, GRAV_PHI>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        else if (defer) kern<true, GRAV_NONE>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        else if (grav) kern<false, GRAV_PHI>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        else kern<false, GRAV_NONE>()<<<grid, b, smem(), s>>>(inst, work, nwork, src, dst, dt, active);
        return cudaGetLastError();
    }
};

template <class T, int K = 0> struct ShapeLoop {
    static cudaError_t prepare() {
        if constexpr (K < BatchShapes<T>::N) {
            cudaError_t e = ShapeOps<T, K>::prepare();
            if (e != cudaSuccess) return e;
            return ShapeLoop<T, K + 1>::prepare();
        }
        return cudaSuccess;
    }
    static TileShape shape(int k) {
        if constexpr (K < BatchShapes<T>::N) {
            if (k == K) return TileShape{ShapeOps<T, K>::S::TX, ShapeOps<T, K>::S::TY};
            return ShapeLoop<T, K + 1>::shape(k);
        }
        return TileShape{0, 0};
    }
    static cudaError_t resident(int k, int* per_sm) {
        if constexpr (K < BatchShapes<T>::N) {
            if (k == K) return ShapeOps<T, K>::resident(per_sm);
            return ShapeLoop<T, K + 1>::resident(k, per_sm);
        }
        return cudaErrorInvalidValue;
    }
    static cudaError_t stage(int k, int grid, const BatchInst<T>* inst, const int2* work, int nwork, int src, int dst,
                             bool defer, bool grav, const double* dt, const int* active, cudaStream_t s) {
        if constexpr (K < BatchShapes<T>::N) {
            if (k == K) return ShapeOps<T, K>::stage(grid, inst, work, nwork, src, dst, defer, grav, dt, active, s);
            return ShapeLoop<T, K + 1>::stage(k, grid, inst, work, nwork, src, dst, defer, grav, dt, active, s);
        }
        return cudaErrorInvalidValue;
    }
};

// one warp per reduce tile, RWPB tiles per CTA
inline int rgrid(int nrwork) { return nrwork < 1 ? 1 : (nrwork + RWPB - 1) / RWPB; }

}  // namespace

template <class T>
cudaError_t BatchLaunch<T>::stage_rec(const BatchInst<T>* inst, const int2* work, int nwork, int src, int dst,
                                      bool defer, bool grav, const double* dt, const int* active, cudaStream_t s) {
    static bool prepared = false;
    if (!prepared) {
        cudaError_t e = ShapeOps<T, 0>::prepare_rec();
        if (e != cudaSuccess) return e;
        prepared = true;
    }
    return ShapeOps<T, 0>::stage_rec(nwork < 1 ? 1 : nwork, inst, work, nwork, src, dst, defer, grav, dt, active, s);
}

template <class T> int BatchLaunch<T>::n_shapes() { return BatchShapes<T>::N; }
template <class T> TileShape BatchLaunch<T>::shape(int k) { return ShapeLoop<T>::shape(k); }
template <class T> cudaError_t BatchLaunch<T>::prepare() { return ShapeLoop<T>::prepare(); }
template <class T> cudaError_t BatchLaunch<T>::resident(int k, int* per_sm) { return ShapeLoop<T>::resident(k, per_sm); }

template <class T>
cudaError_t BatchLaunch<T>::stage(int k, int grid, const BatchInst<T>* inst, const int2* work, int nwork, int src,
                                  int dst, bool defer, bool grav, const double* dt, const int* active,
                                  cudaStream_t s) {
    return ShapeLoop<T>::stage(k, grid, inst, work, nwork, src, dst, defer, grav, dt, active, s);
}

template <class T>
cudaError_t BatchLaunch<T>::average(const BatchInst<T>* inst, const int2* rwork, int nrwork, int a, int d, int b,
                                    const double* dt, const int* active, double* spd_part, double* rho_part,
                                    cudaStream_t s) {
    m2b_average_kernel<T><<<rgrid(nrwork), RNT, 0, s>>>(inst, rwork, nrwork, a, d, b, dt, active, spd_part, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t BatchLaunch<T>::speeds(const BatchInst<T>* inst, const int2* rwork, int nrwork, int src,
                                   double* spd_part, double* rho_part, cudaStream_t s) {
    m2b_speed_kernel<T><<<rgrid(nrwork), RNT, 0, s>>>(inst, rwork, nrwork, src, spd_part, rho_part);
    return cudaGetLastError();
}

template <class T>
cudaError_t BatchLaunch<T>::rho_sum(const BatchInst<T>* inst, const int2* rwork, int nrwork, int src,
                                    const int* active, double* rho_part, cudaStream_t s) {
    m2b_rho_sum_kernel<T><<<rgrid(nrwork), RNT, 0, s>>>(inst, rwork, nrwork, src, active, rho_part);
    return cudaGetLastError();
}

}  // namespace ccb
