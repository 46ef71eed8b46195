// C ABI of the batched 2D MHD ensemble (include/cc_batch.h).
//
// Per step, for all instances at once (each instance's step is the
// single-grid step of capi.cu, M2:1111-1117 and 838-869):
//   [gravity]  density means (finaliser) -> direct Poisson(U^n.rho) -> phi
//   finaliser: dt_i from the CFL partials, clamped to t_end_i; active_i
//   stage 1:   persistent stage kernel over the stage work-list, U^n -> S1
//   [gravity]  density partials of S1 -> means -> direct Poisson(S1.rho) -> phi
//   stage 2:   Joule(S1) -> S2 (deferred Joule, as on the single grid)
//   average:   U^{n+1} = floors(0.5 (U^n + Joule(S2))) + CFL/density partials
//   clock:     t_i += dt_i for active instances
// The rotation of the three state buffers is shared; three steps are one
// CUDA graph.
#include <memory>

#include "batch_host.h"

using namespace ccb;

namespace {

struct BatchHandle : cc_handle {
    std::unique_ptr<BatchBase> impl;
};

BatchBase* bt(cc_handle* h) {
    if (!h || h->kind != KIND_BATCH) return nullptr;
    return static_cast<BatchHandle*>(h)->impl.get();
}

}  // namespace

extern "C" {

int cc_batch_create(const cc_mhd2d_params* params, int n, cc_handle** out) {
    if (!params || !out || n < 1) return CC_ERR_ARG;
    *out = nullptr;
    const int prec = params[0].precision;
    if (prec != CC_FP64 && prec != CC_FP32) return CC_ERR_ARG;
    auto h = std::make_unique<BatchHandle>();
    h->kind = KIND_BATCH;
    for (int i = 0; i < n; i++) {
        const cc_mhd2d_params& q = params[i];
        std::string where = "instance " + std::to_string(i) + ": ";
        int code = CC_OK;
        if (q.precision != prec) { code = CC_ERR_ARG; where += "all instances must share one precision"; }
        else if (q.Nx < 4 || q.Ny < 4) { code = CC_ERR_ARG; where += "Nx and Ny must be >= 4"; }
        else if (q.Nx > 65535 * 16 || q.Ny > 65535 * 8) { code = CC_ERR_ARG; where += "grid too large"; }
        else if (!(q.x1 > q.x0) || !(q.y1 > q.y0)) { code = CC_ERR_ARG; where += "empty domain"; }
        else if (q.compensated) { code = CC_ERR_UNSUPPORTED; where += "the ensemble has no compensated update"; }
        else if (q.gravity_on && q.poisson_kind != CC_POISSON_DIRECT) {
            code = CC_ERR_UNSUPPORTED;
            where += "instances with gravity need poisson_kind == CC_POISSON_DIRECT";
        } else if (q.gravity_on && (q.Nx > CC_BATCH_MAX_DIRECT_SIDE || q.Ny > CC_BATCH_MAX_DIRECT_SIDE)) {
            code = CC_ERR_UNSUPPORTED;
            where += "direct Poisson side above CC_BATCH_MAX_DIRECT_SIDE";
        }
        if (code != CC_OK) {
            h->err = where;
            *out = h.release();
            return code;
        }
    }
    if (cudaGetDevice(&h->device) != cudaSuccess) return CC_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return CC_ERR_CUDA;
    h->stream = h->own;
    if (prec == CC_FP64) h->impl = std::make_unique<Batch<double>>(h.get(), params, n);
    else h->impl = std::make_unique<Batch<float>>(h.get(), params, n);
    int r = h->impl->init();
    *out = h.release();
    return r;
}

int cc_batch_upload(cc_handle* h, int inst, const double* const* f) {
    BatchBase* b = bt(h);
    if (!b) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return b->upload(inst, f);
}

int cc_batch_download(cc_handle* h, int inst, double* const* f) {
    BatchBase* b = bt(h);
    if (!b) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return b->download(inst, f);
}

int cc_batch_compute_dt(cc_handle* h, double* dt) {
    BatchBase* b = bt(h);
    if (!b || !dt) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return b->compute_dt(dt);
}

int cc_batch_advance(cc_handle* h, int nsteps, double* t) {
    BatchBase* b = bt(h);
    if (!b) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return b->advance(nsteps, t);
}

int cc_batch_diagnostics(cc_handle* h, int inst, cc_diag* d) {
    BatchBase* b = bt(h);
    if (!b) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return b->diagnostics(inst, d);
}

int cc_batch_times(cc_handle* h, double* t) {
    BatchBase* b = bt(h);
    if (!b || !t) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return b->times(t);
}

int cc_batch_autotune(cc_handle* h, int reps, int* shape, double* ms) {
    BatchBase* b = bt(h);
    if (!b) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return b->autotune(reps, shape, ms);
}

int cc_batch_set_shape(cc_handle* h, int shape) {
    BatchBase* b = bt(h);
    if (!b) return CC_ERR_ARG;
    return b->set_shape(shape);
}

int cc_batch_get_info(cc_handle* h, cc_batch_info* info) {
    BatchBase* b = bt(h);
    if (!b || !info) return CC_ERR_ARG;
    return b->info(info);
}

}  // extern "C"
