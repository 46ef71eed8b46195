// C ABI of the discrete adjoint of the 2D MHD step (include/cc_adjoint.h); the
// adjoint itself is adjoint_impl.cuh.  This unit holds the FP64 instantiation
// (built with -fmad=false, so that its reverse kernels recompute the FP64
// forward's intermediates bit for bit); the FP32 one is adjoint_f32.cu.
#include <memory>

#include "adjoint_impl.cuh"

using namespace ccb;

namespace ccb {
extern template struct Adjoint<float>;
template struct Adjoint<double>;
}  // namespace ccb

namespace {

struct AdjHandle : cc_handle {
    std::unique_ptr<AdjointBase> impl;
};

AdjointBase* aj(cc_handle* h) {
    if (!h || h->kind != KIND_ADJOINT) return nullptr;
    return static_cast<AdjHandle*>(h)->impl.get();
}

}  // namespace

extern "C" {

int cc_adjoint_create(const cc_mhd2d_params* p, int checkpoint_every, int max_steps, cc_handle** out) {
    if (!p || !out) return CC_ERR_ARG;
    *out = nullptr;
    auto h = std::make_unique<AdjHandle>();
    h->kind = KIND_ADJOINT;
    std::string why;
    int code = CC_OK;
    if (p->precision != CC_FP64 && p->precision != CC_FP32) { code = CC_ERR_ARG; why = "unknown precision"; }
    else if (p->compensated) { code = CC_ERR_UNSUPPORTED; why = "the adjoint has no compensated update"; }
    else if (checkpoint_every < 1 || max_steps < 1) { code = CC_ERR_ARG; why = "checkpoint_every and max_steps must be >= 1"; }
    else if (p->Nx < 4 || p->Ny < 4 || !(p->x1 > p->x0) || !(p->y1 > p->y0)) { code = CC_ERR_ARG; why = "bad grid"; }
    else if (p->gravity_on && p->poisson_kind != CC_POISSON_DIRECT && p->poisson_kind != CC_POISSON_SOR) {
        code = CC_ERR_UNSUPPORTED;
        why = "gravity needs poisson_kind CC_POISSON_DIRECT or CC_POISSON_SOR";
    } else if (p->gravity_on && p->poisson_kind == CC_POISSON_SOR &&
               ((p->periodic_x && (p->Nx & 1)) || (p->periodic_y && (p->Ny & 1)))) {
        code = CC_ERR_UNSUPPORTED;
        why = "red-black SOR needs an even extent along periodic axes";
    } else if (p->gravity_on && (p->Nx > CC_BATCH_MAX_DIRECT_SIDE || p->Ny > CC_BATCH_MAX_DIRECT_SIDE)) {
        code = CC_ERR_UNSUPPORTED;
        why = "direct Poisson side above CC_BATCH_MAX_DIRECT_SIDE";
    }
    if (code != CC_OK) {
        h->err = why;
        *out = h.release();
        return code;
    }
    if (cudaGetDevice(&h->device) != cudaSuccess) return CC_ERR_CUDA;
    if (cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking) != cudaSuccess) return CC_ERR_CUDA;
    h->stream = h->own;
    cc_mhd2d_params q = *p;
    q.t_end = 1e300;   // the run length is the caller's step count
    if (q.precision == CC_FP32)
        h->impl = std::make_unique<Adjoint<float>>(h.get(), q, checkpoint_every, max_steps);
    else
        h->impl = std::make_unique<Adjoint<double>>(h.get(), q, checkpoint_every, max_steps);
    const int r = h->impl->init_adjoint();
    *out = h.release();
    return r;
}

int cc_adjoint_upload(cc_handle* h, const double* const* f) {
    AdjointBase* a = aj(h);
    if (!a || !f) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->upload0(f);
}

int cc_adjoint_forward(cc_handle* h, int nsteps, double t0, int replay, double* t_out) {
    AdjointBase* a = aj(h);
    if (!a) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->forward(nsteps, t0, replay, t_out);
}

int cc_adjoint_download(cc_handle* h, double* const* f) {
    AdjointBase* a = aj(h);
    if (!a || !f) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->download_final(f);
}

int cc_adjoint_get_dts(cc_handle* h, double* dts, int n) {
    AdjointBase* a = aj(h);
    if (!a || !dts || n < 0) return CC_ERR_ARG;
    if (n > a->nrec) return fail(h, CC_ERR_ARG, "fewer recorded steps than requested");
    for (int i = 0; i < n; i++) dts[i] = a->dts[i];
    return CC_OK;
}

int cc_adjoint_set_dts(cc_handle* h, const double* dts, int n) {
    AdjointBase* a = aj(h);
    if (!a || !dts) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->set_dts(dts, n);
}

int cc_adjoint_vjp(cc_handle* h, const double* const* lam_final, double* const* lam_initial, double* lam_eta) {
    AdjointBase* a = aj(h);
    if (!a || !lam_final) return CC_ERR_ARG;
    if (int r = set_dev(h)) return r;
    return a->vjp(lam_final, lam_initial, lam_eta);
}

}  // extern "C"
