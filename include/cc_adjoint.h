/*
 * cc_adjoint.h -- discrete adjoint (vector-Jacobian product) of n steps of the
 * 2D resistive-MHD step (mhd2d_resistive_hlld_ct_gravity.cpp, rk2_step
 * M2:838-869 with compute_dt M2:579-598), one grid, FP64 or FP32.
 *
 * No reference counterpart: the reference has no derivatives.  The forward
 * map is the step of cc_batch.h / cc_step.h: RK2 stages of MUSCL-MC + HLLD +
 * CT + resistive EMF + gravity kick + Joule/Bz diffusion, floors, RK
 * average; with gravity on, the Poisson solve is the direct solve
 * (CC_POISSON_DIRECT) or the red-black SOR (CC_POISSON_SOR).  Each step's dt is computed by the CFL rule in the
 * recorded forward run and then treated as a constant (replayed in the
 * recomputation and in any finite-difference check); the derivative of a
 * floor, limiter or Riemann-solver branch is that of the branch taken.
 *
 * Use: cc_adjoint_upload(U0) ; cc_adjoint_forward(n, t0, 0, &t) records dt and
 * keeps a checkpoint every `checkpoint_every` steps ; cc_adjoint_download
 * gives U_n ; cc_adjoint_vjp(lambda_n) returns lambda_0 = (dU_n/dU_0)^T
 * lambda_n and d(lambda_n . U_n)/d eta.  cc_adjoint_forward(n, t0, 1, ...)
 * reruns the forward with the recorded dt (for finite differences).
 * State and adjoint arrays: f = {rho, mx, my, mz, E, Bz, Bx_f, By_f} in the
 * reference layouts (cc_step.h).
 */
#ifndef CC_ADJOINT_H
#define CC_ADJOINT_H

#include "cc_step.h"

#ifdef __cplusplus
extern "C" {
#endif

/* p: precision CC_FP64, or CC_FP32 (an FP32 forward run reversed by the same
 * kernels in FP32, eta's adjoint summed in FP64; states and adjoints cross
 * the API as FP64 arrays); with gravity_on, poisson_kind is CC_POISSON_DIRECT
 * (the direct solve, its own adjoint) or CC_POISSON_SOR (the red-black SOR
 * of cc_mhd2d_*, sor_iters sweeps or the tolerance; reversed with the sweep
 * count each solve took; even extents along periodic axes); compensated must
 * be 0.  Device
 * memory: about 40 planes of (Nx+1)*(Ny+1) values per step of a checkpoint
 * block, plus 8 planes per checkpoint of max_steps. */
int cc_adjoint_create(const cc_mhd2d_params* p, int checkpoint_every, int max_steps, cc_handle** out);
int cc_adjoint_upload(cc_handle* h, const double* const* f);
/* replay = 0: dt from the CFL rule, recorded; 1: the recorded dt of a previous run. */
int cc_adjoint_forward(cc_handle* h, int nsteps, double t0, int replay, double* t_out);
/* state after the last forward run */
int cc_adjoint_download(cc_handle* h, double* const* f);
/* the first n recorded dt values */
int cc_adjoint_get_dts(cc_handle* h, double* dts, int n);
/* make dts[0..n) the recorded sequence (a replayed forward run and the next
 * vjp use it), e.g. to rerun another handle's run with a perturbed parameter */
int cc_adjoint_set_dts(cc_handle* h, const double* dts, int n);
/* lam_final: adjoint of the final state (8 arrays); lam_initial (8 arrays, may
 * be NULL) and lam_eta (may be NULL) receive the adjoints of the initial state
 * and of eta along the trajectory of the last forward run (recorded or
 * replayed), with the recorded dt sequence. */
int cc_adjoint_vjp(cc_handle* h, const double* const* lam_final, double* const* lam_initial, double* lam_eta);

#ifdef __cplusplus
}
#endif

#endif /* CC_ADJOINT_H */
