// The opaque cc_handle shared by every solver's C-ABI implementation, plus
// the error helpers used by them.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../include/cc_step.h"

namespace ccb {
cudaError_t launch_set_scalar(double* p, double v, cudaStream_t s);
}

struct cc_handle {
    int kind = 0;
    int device = 0;
    std::string err;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    cc_perf perf{};
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> timed;  // event pairs around stage launches
    virtual ~cc_handle() {
        for (auto& e : timed) { cudaEventDestroy(e.first); cudaEventDestroy(e.second); }
        if (own) cudaStreamDestroy(own);
    }
    // fold the recorded event pairs into perf.stage_ms (stream must be idle)
    cudaError_t collect() {
        for (auto& e : timed) {
            float ms = 0.f;
            cudaError_t r = cudaEventElapsedTime(&ms, e.first, e.second);
            if (r != cudaSuccess) return r;
            perf.stage_ms += ms;
            perf.stage_launches += 1;
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        timed.clear();
        return cudaSuccess;
    }
};


inline int fail(cc_handle* h, int code, const std::string& msg) {
    if (h) h->err = msg;
    return code;
}

#define CC_CUDA(call)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess)                                                                 \
            return fail(this_handle(), CC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

constexpr int KIND_MHD2D = 1;
constexpr int KIND_MHD3D = 2;
constexpr int KIND_EULER2D = 3;
constexpr int KIND_NS2D = 4;

inline int set_dev(cc_handle* h) {
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) return fail(h, CC_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return CC_OK;
}
