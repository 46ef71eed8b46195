/*
 * cc_step.h -- C ABI of the B200 finite-volume step (libcc_b200.so).
 *
 * The reference solvers have no FFI: each is one C++ translation unit whose
 * main() calls a handful of static functions on std::vector<double> state.
 * Every entry point below replaces one of those calls (cited as file:line in
 * the reference tree) so that a host main() can swap its CPU step for this
 * library without changing its initial conditions, time loop or output.
 *
 * Conventions
 *   - Every function returns an int status: CC_OK (0) or a negative CC_ERR_*.
 *     cc_last_error() gives a message for the last failure on a handle.
 *   - Host arrays are caller-owned FP64 arrays in the reference layouts:
 *       2D cells    q = j*Nx + i                       (Nx*Ny)
 *       2D Bx faces f = j*(Nx+1) + i_face              ((Nx+1)*Ny)
 *       2D By faces f = j_face*Nx + i                  (Nx*(Ny+1))
 *       3D cells    q = (k*Ny + j)*Nx + i
 *       3D faces    Bx (k*Ny+j)*(Nx+1)+i, By (k*(Ny+1)+j)*Nx+i, Bz (k*Ny+j)*Nx+i with k in [0,Nz]
 *     Device copies are owned by the handle; the state stays resident on the
 *     GPU between calls.  Host<->device copies happen only in upload/download
 *     and in calls that take or return host arrays.
 *   - A handle owns one CUDA stream and is used by one host thread at a time.
 *   - precision: CC_FP64 runs every kernel in double precision and is the
 *     parity path; CC_FP32 runs the flux/EMF/update bulk in single precision
 *     with FP64 reductions (dt minimum, conserved sums, Poisson residual).
 */
#ifndef CC_STEP_H
#define CC_STEP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define CC_OK                 0
#define CC_ERR_ARG           -1   /* bad argument (null pointer, size, enum) */
#define CC_ERR_CUDA          -2   /* a CUDA runtime call failed */
#define CC_ERR_STATE         -3   /* call not valid in the handle's state */
#define CC_ERR_NONFINITE     -4   /* dt not finite or <= 0 (euler2d_gravity_hllc.cpp:699-702) */
#define CC_ERR_NOT_CONVERGED -5   /* Poisson SOR hit its iteration cap before sor_tol */
#define CC_ERR_UNSUPPORTED   -6   /* option combination not implemented */

/* ---- enums ---- */
#define CC_FP64 0
#define CC_FP32 1

#define CC_POISSON_SOR 0   /* red-black SOR (GPU-parallel ordering of M2's SOR) */
#define CC_POISSON_FFT 1   /* spectral periodic solve, power-of-two grids */
#define CC_POISSON_DIRECT 2 /* exact solve of the SOR's discrete problem (batched ensemble, cc_batch.h) */
#define CC_GRAVITY_ENCLOSED 3 /* Euler/HLLC only: enclosed-mass radial gravity, compute_enclosed_mass_gravity
                                 (euler2d_gravity_hllc.cpp:226-286, the rhs's commented-out alternative, EH:411) */
#define CC_GRAVITY_SHELLS 4   /* Euler/HLLC only: radial gravity from cell masses binned into Nr_bins radial
                                 shells about (xc, yc), gravity_accel_from_enclosed_mass
                                 (gravity_enclosed.h:18-96) */
#define CC_POISSON_SOR_LEX 5 /* 2D MHD: the reference's lexicographic SOR (M2:178-237) in its own sweep order,
                                with its sequential density and phi means: the same phi bit for bit (FP64).
                                A parity mode for drop-in runs: one CTA, nx+ny-1 barriers and an N-term
                                sequential sum per sweep */

typedef struct cc_handle cc_handle;

/*
 * 2D resistive MHD + self-gravity.  Fields mirror Params in
 * mhd2d_resistive_hlld_ct_gravity.cpp:44-86 (IC knobs omitted: initial
 * conditions are host-side); the last four fields are additions.
 */
typedef struct cc_mhd2d_params {
    double gamma;
    double cfl;
    double x0, x1, y0, y1;
    int32_t Nx, Ny;
    double t_end;
    double dt_store;
    double floor_rho;
    double floor_P;
    int32_t periodic_x;     /* 1: periodic (imod); 0: outflow (clamp)      */
    int32_t periodic_y;
    double eta;             /* constant resistivity                         */
    int32_t gravity_on;
    double G;
    double softening;       /* unused by the Poisson path, kept for layout  */
    int32_t sor_iters;      /* sweep count (sor_tol <= 0) or sweep cap      */
    double sor_omega;
    /* additions */
    double sor_tol;         /* > 0: stop once max|lap(phi)-rhs| < sor_tol   */
    int32_t poisson_kind;   /* CC_POISSON_SOR or CC_POISSON_FFT             */
    int32_t precision;      /* CC_FP64 or CC_FP32                           */
    int32_t compensated;    /* FP32 only, 1: compensated (Kahan-style) state
                               update -- every state plane carries its FP32
                               rounding residual, each stage increment and
                               the RK average are added with an error-free
                               sum; uploads split FP64 values into value +
                               residual, downloads return their sum.  The
                               batched ensemble and the adjoint reject it. */
} cc_mhd2d_params;

/*
 * 3D resistive MHD with the hybrid cold+thermal EOS.  Fields mirror Params in
 * mhd3d_resistive_hlld_ct.cpp:43-89 (IC knobs omitted).
 */
typedef struct cc_mhd3d_params {
    double gamma1, gamma2, K1, rho_nuc, gamma_th;
    double rho_bounce, gamma_bounce, Kbounce;
    double gamma_init;
    double cfl;
    double x0, x1, y0, y1, z0, z1;
    int32_t Nx, Ny, Nz;
    int32_t precision;      /* addition: CC_FP64 or CC_FP32 */
    double t_end;
    double dt_store;
    double floor_rho;
    double floor_P;
    int32_t periodic_x, periodic_y, periodic_z;
    int32_t reserved;
    double eta;
} cc_mhd3d_params;

/*
 * 2D Euler + self-gravity with HLLC.  Fields mirror Params in
 * euler2d_gravity_hllc.cpp:29-56; the SOR constants that the reference
 * hard-codes inside its Poisson solve (euler2d_gravity_hllc.cpp:329-331) are
 * fields here.
 */
typedef struct cc_euler2d_params {
    double gamma;
    double cfl;
    double x0, x1, y0, y1;
    int32_t Nx, Ny;
    double t_end;
    double dt_store;
    double floor_rho;
    double floor_P;
    int32_t periodic_x, periodic_y;
    int32_t gravity_on;
    int32_t sor_max_iter;   /* 50000 in the reference */
    double G;
    double softening;
    double sor_tol;         /* 1e-10 */
    double sor_omega;       /* 1.7   */
    int32_t poisson_kind;   /* addition */
    int32_t precision;      /* addition */
    /* the shell-binned provider's knobs (CC_GRAVITY_SHELLS; Params of the
       solver that includes gravity_enclosed.h, euler2d_h5.cpp:42-45) */
    int32_t Nr_bins;        /* 512: radial shells (at least 8 are used)    */
    int32_t reserved;
    double xc, yc;          /* 0.5, 0.5: gravity centre                     */
} cc_euler2d_params;

/*
 * 2D compressible Navier-Stokes (explicit viscosity) + periodic spectral
 * self-gravity with first-order HLLC.  Fields mirror Params in
 * navier_stokes_2d_hllc_poisson.cpp:53-85 (the HDF5 file name excepted);
 * periodic in both directions (NS:32), Nx and Ny powers of two when
 * gravity_on (NS:614-617).
 */
typedef struct cc_ns2d_params {
    double gamma;
    double cfl;
    double x0, x1, y0, y1;
    int32_t Nx, Ny;
    double t_end;
    double dt_store;
    uint32_t seed;          /* 42: std::mt19937 seed of the reference IC */
    int32_t viscosity_on;
    double floor_rho;
    double floor_P;
    double mu;              /* dynamic viscosity, 1e-6 */
    double cfl_visc;        /* explicit-diffusion CFL, 0.05 */
    int32_t gravity_on;
    int32_t precision;      /* addition */
    double G;
} cc_ns2d_params;

/* Diagnostics gathered on the device (FP64 sums over cells). */
typedef struct cc_diag {
    double mass;            /* sum rho * dV        */
    double mom_x, mom_y, mom_z;
    double energy;          /* sum E * dV          */
    double max_divB;        /* max |div B| over cells (M2:873-879) */
    double t;               /* simulated time advanced by cc_*_advance */
    double dt_last;         /* last dt used        */
    int64_t steps;          /* steps taken by cc_*_advance */
    int32_t poisson_iters;  /* sweeps of the last SOR solve (0 for FFT) */
    int32_t nonfinite;      /* 1 if a non-finite conserved value was seen */
    double poisson_residual;/* max |lap(phi)-rhs| after the last SOR solve */
} cc_diag;

/* Performance counters of a handle (no reference counterpart: measurement
 * support).  kernel_launches counts every kernel this library launched on the
 * handle (graph replays included).  With profiling on, the stage kernels are
 * bracketed by CUDA events on the handle's stream and time loops run without
 * graphs; stage_ms is their summed event time. */
typedef struct cc_perf {
    int64_t kernel_launches;
    int64_t stage_launches;     /* stage-kernel launches that were event-timed */
    double stage_ms;            /* summed event time of those launches */
    int64_t poisson_solves;
    int64_t steps;
} cc_perf;

/* Fill with the reference defaults (mhd2d_resistive_hlld_ct_gravity.cpp:44-86). */
void cc_mhd2d_params_default(cc_mhd2d_params* p);

/* ---- handle lifetime (all solvers) ---- */
int cc_mhd2d_create(const cc_mhd2d_params* p, cc_handle** out);
int cc_destroy(cc_handle* h);
const char* cc_last_error(const cc_handle* h);
/* Make the handle issue its work on a caller stream (cudaStream_t as void*);
 * NULL restores the handle's own stream. */
int cc_set_stream(cc_handle* h, void* stream);
int cc_synchronize(cc_handle* h);

/* Measurement support (no reference counterpart). */
int cc_set_profiling(cc_handle* h, int on);
int cc_get_perf(cc_handle* h, cc_perf* out);   /* synchronizes the handle's stream */
int cc_reset_perf(cc_handle* h);

/* ---- 2D MHD state transfer (reference layouts, FP64 host arrays) ---- */
/* Ucc {rho,mx,my,mz,E,Bz} and Bfaces {Bx_f,By_f}: M2:88-95 */
int cc_mhd2d_upload(cc_handle* h,
                    const double* rho, const double* mx, const double* my,
                    const double* mz, const double* E, const double* Bz,
                    const double* Bx_f, const double* By_f);
int cc_mhd2d_download(cc_handle* h,
                      double* rho, double* mx, double* my,
                      double* mz, double* E, double* Bz,
                      double* Bx_f, double* By_f);

/* ---- 2D MHD step pieces (each replaces one reference call) ---- */

/* compute_poisson_gravity_periodic(p, U.rho, dx, dy) -> GravField
 * (mhd2d_resistive_hlld_ct_gravity.cpp:178-237).  Solves on the resident rho
 * and keeps g on the device; gx/gy (Nx*Ny each) may be NULL, otherwise g is
 * also copied to the host.  With gravity_on == 0, g is zero. */
int cc_mhd2d_compute_gravity(cc_handle* h, double* gx, double* gy);

/* compute_dt(p, U, B, dx, dy) (mhd2d_resistive_hlld_ct_gravity.cpp:579-598).
 * FP64 max-reduction of |u|+c_f over cells; writes dt to *dt (host). */
int cc_mhd2d_compute_dt(cc_handle* h, double* dt);

/* rk2_step(p, U, B, g, dx, dy, dt) (mhd2d_resistive_hlld_ct_gravity.cpp:838-869).
 * gx/gy: host gravity arrays for stage 1, or NULL to use the device-resident g
 * from the last cc_mhd2d_compute_gravity.  Stage 2 always solves Poisson on the
 * stage-1 density on the device (M2:843). */
int cc_mhd2d_rk2_step(cc_handle* h, const double* gx, const double* gy, double dt);

/* The body of the main() time loop (mhd2d_resistive_hlld_ct_gravity.cpp:1111-1117)
 * run nsteps times on the device: g = Poisson(rho); dt = compute_dt;
 * dt = min(dt, t_end - t); rk2_step.  Stops early once t >= t_end.  *t is the
 * current time on entry and the advanced time on return (may be NULL: start at
 * the handle's clock).  dt never leaves the device. */
int cc_mhd2d_advance(cc_handle* h, int nsteps, double* t);

/* Choice of the stage kernel (no counterpart in the reference, whose
 * advance_stage M2:690-834 is one function): CC_STAGE_TILE, the default, one
 * CTA per tile of cells with a recomputed halo (the only form for FP64), or
 * CC_STAGE_MARCH, FP32 only, a CTA per column strip that
 * marches up a segment of seg_rows rows carrying the rows below it (0: a
 * length chosen from the grid so the segments fill the GPU).  Both evaluate
 * the same expressions; a tuning and testing switch. */
#define CC_STAGE_TILE 0
#define CC_STAGE_MARCH 1
int cc_mhd2d_set_stage_kernel(cc_handle* h, int kind, int seg_rows);

/* Diagnostics of the resident state. */
int cc_mhd2d_diagnostics(cc_handle* h, cc_diag* d);

/* The derived fields the reference main() stores at each snapshot
 * (mhd2d_resistive_hlld_ct_gravity.cpp:1065-1106) from the resident state:
 * out[0..9] = rho, P, Mach, u, v, vabs, Bx, By, Bz, divB, each Nx*Ny doubles
 * (row-major, x fastest); a NULL entry is skipped.  Bx, By are the cell-centred
 * averages of the faces; FP64 handles give the reference's values bit for bit.
 * The first call allocates 10*Nx*Ny doubles of device scratch for the handle. */
int cc_mhd2d_derived(cc_handle* h, double* const* out);

/* Checkpoint / restart (no counterpart in the reference, which keeps no
 * restart file).  save: the resident state in the reference layouts as FP64,
 * the clock (t, steps) and the parameters, into one file at path: magic
 * "CCB2DCK1", version, precision, Nx, Ny, the cc_mhd2d_params bytes, t, steps,
 * the 8 arrays, then an FNV-1a 64-bit checksum of all preceding bytes.  load:
 * into a handle whose grid, domain, boundaries and precision equal the file's
 * (other parameters, e.g. t_end, may differ); restores state and clock, so a
 * run continued from a checkpoint matches the uninterrupted run bit for bit.
 * Errors: CC_ERR_IO (open, read, write), CC_ERR_ARG (bad magic, version,
 * checksum or a grid mismatch). */
#define CC_ERR_IO -8
int cc_mhd2d_checkpoint_save(cc_handle* h, const char* path);
int cc_mhd2d_checkpoint_load(cc_handle* h, const char* path);

/* ---- 3D MHD (mhd3d_resistive_hlld_ct.cpp) ---- */

/* Fill with the reference defaults (mhd3d_resistive_hlld_ct.cpp:43-89). */
void cc_mhd3d_params_default(cc_mhd3d_params* p);
int cc_mhd3d_create(const cc_mhd3d_params* p, cc_handle** out);
/* Ucc {rho,mx,my,mz,E} and Bfaces {Bx_f,By_f,Bz_f}: M3:91-99 */
int cc_mhd3d_upload(cc_handle* h, const double* rho, const double* mx, const double* my, const double* mz,
                    const double* E, const double* Bx_f, const double* By_f, const double* Bz_f);
int cc_mhd3d_download(cc_handle* h, double* rho, double* mx, double* my, double* mz, double* E,
                      double* Bx_f, double* By_f, double* Bz_f);
/* compute_dt(p, U, B, dx, dy, dz) (mhd3d_resistive_hlld_ct.cpp:626-648) */
int cc_mhd3d_compute_dt(cc_handle* h, double* dt);
/* rk2_step(p, U, B, dx, dy, dz, dt) (mhd3d_resistive_hlld_ct.cpp:1034-1066) */
int cc_mhd3d_rk2_step(cc_handle* h, double dt);
/* nsteps of the main() loop body (mhd3d_resistive_hlld_ct.cpp:1285-1291) on the
 * device: dt = compute_dt, clamped to t_end; rk2_step.  Stops once t >= t_end. */
int cc_mhd3d_advance(cc_handle* h, int nsteps, double* t);
/* FP64 sums and max |div B| (mhd3d_resistive_hlld_ct.cpp:1070-1078) */
int cc_mhd3d_diagnostics(cc_handle* h, cc_diag* d);
/* The fields the reference main() stores per snapshot (mhd3d_resistive_hlld_ct.cpp:1293-1321):
 * out[0..10] = rho, P, Mach, u, v, w, vabs, Bx, By, Bz, divB (Nx*Ny*Nz doubles
 * each, x fastest; NULL entries skipped); B cell-centred from the faces,
 * Mach with the hybrid-EOS sound speed.  The first call allocates
 * 11*Nx*Ny*Nz doubles of device scratch for the handle. */
int cc_mhd3d_derived(cc_handle* h, double* const* out);
/* Restart files of the 3D handle: {rho, mx, my, mz, E, Bx_f, By_f, Bz_f}, the
 * clock and the parameters (as cc_euler2d_checkpoint_*, magic "CCM3DCK1"). */
int cc_mhd3d_checkpoint_save(cc_handle* h, const char* path);
int cc_mhd3d_checkpoint_load(cc_handle* h, const char* path);

/* ---- 2D Euler + self-gravity, HLLC (euler2d_gravity_hllc.cpp) ---- */

/* Fill with the reference defaults (euler2d_gravity_hllc.cpp:29-56, 329-331). */
void cc_euler2d_params_default(cc_euler2d_params* p);
int cc_euler2d_create(const cc_euler2d_params* p, cc_handle** out);
/* State {rho,mx,my,E}: EH:58-60 */
int cc_euler2d_upload(cc_handle* h, const double* rho, const double* mx, const double* my, const double* E);
int cc_euler2d_download(cc_handle* h, double* rho, double* mx, double* my, double* E);
/* compute_dt(p, U) (euler2d_gravity_hllc.cpp:390-404) */
int cc_euler2d_compute_dt(cc_handle* h, double* dt);
/* compute_poisson_gravity_periodic(p, U) (euler2d_gravity_hllc.cpp:288-386) on the
 * resident state; gx/gy (Nx*Ny) may be NULL. */
int cc_euler2d_compute_gravity(cc_handle* h, double* gx, double* gy);
/* rk2_step(p, U, dt) (euler2d_gravity_hllc.cpp:529-550); the right-hand side
 * solves Poisson itself, on U and on the stage-1 state (EH:411). */
int cc_euler2d_rk2_step(cc_handle* h, double dt);
/* nsteps of the main() loop body (euler2d_gravity_hllc.cpp:697-706) on the
 * device; returns CC_ERR_NONFINITE if dt is not finite or not positive (where
 * the reference aborts, EH:699-702), the state then being the last good one. */
int cc_euler2d_advance(cc_handle* h, int nsteps, double* t);
int cc_euler2d_diagnostics(cc_handle* h, cc_diag* d);
/* The fields the reference main() stores per snapshot (euler2d_gravity_hllc.cpp:661-689):
 * out[0..2] = rho, P, Mach (Nx*Ny doubles each; NULL entries skipped), from a
 * floored copy of each cell; Mach = |v| / a, 0 where a <= 0.  The first call
 * allocates 3*Nx*Ny doubles of device scratch for the handle. */
int cc_euler2d_derived(cc_handle* h, double* const* out);
/* Restart files of the Euler handle: state {rho, mx, my, E}, the clock and the
 * parameters in one checksummed file (layout in csrc/checkpoint.h, magic
 * "CCEH2CK1").  No reference counterpart.  Load checks the grid, domain,
 * boundaries and precision against the handle's (CC_ERR_ARG otherwise; a
 * corrupted file: CC_ERR_ARG; an unreadable one: CC_ERR_IO). */
int cc_euler2d_checkpoint_save(cc_handle* h, const char* path);
int cc_euler2d_checkpoint_load(cc_handle* h, const char* path);

/* ---- 2D Navier-Stokes + FFT self-gravity, HLLC (navier_stokes_2d_hllc_poisson.cpp) ---- */

/* Fill with the reference defaults (navier_stokes_2d_hllc_poisson.cpp:53-85). */
void cc_ns2d_params_default(cc_ns2d_params* p);
int cc_ns2d_create(const cc_ns2d_params* p, cc_handle** out);
/* State {rho, rho u, rho v, E} (U4, NS:88-90): Nx*Ny doubles each, q = i + Nx*j */
int cc_ns2d_upload(cc_handle* h, const double* rho, const double* mx, const double* my, const double* E);
int cc_ns2d_download(cc_handle* h, double* rho, double* mx, double* my, double* E);
/* compute_dt(U) (NS:521-546), without the loop's clamp to t_end */
int cc_ns2d_compute_dt(cc_handle* h, double* dt);
/* solve_poisson_periodic_fft + compute_gravity_accel (NS:285-360) on the
 * density of cons_to_prim of the resident state (NS:372-383); phi, gx, gy
 * (Nx*Ny each) may be NULL.  Zero fields with gravity off. */
int cc_ns2d_compute_gravity(cc_handle* h, double* phi, double* gx, double* gy);
/* compute_rhs(U) (NS:363-518) of the resident state: dU[0..3] = the rates of
 * rho, rho u, rho v, E (Nx*Ny doubles each; NULL entries skipped). */
int cc_ns2d_compute_rhs(cc_handle* h, double* const* dU);
/* One SSP-RK2 (Heun) step of the main() loop body (NS:762-781) with this dt. */
int cc_ns2d_rk2_step(cc_handle* h, double dt);
/* nsteps of the main() loop body (NS:758-791) on the device: dt from
 * compute_dt, clamped so that t does not pass t_end; once t >= t_end - 1e-14
 * the remaining steps do nothing.  *t (if not NULL) sets the clock first and
 * receives it after. */
int cc_ns2d_advance(cc_handle* h, int nsteps, double* t);
int cc_ns2d_diagnostics(cc_handle* h, cc_diag* d);
/* The fields the reference main() stores per snapshot (NS:698-746):
 * out[0..7] = rho, P, Mach, u, v, momx, momy, Phi (Nx*Ny doubles each; NULL
 * entries skipped), from cons_to_prim of each cell; Mach = |v| / a, 0 where
 * a <= 0; Phi the spectral potential of the state's density (0 with gravity
 * off).  The first call allocates 8*Nx*Ny doubles of device scratch. */
int cc_ns2d_derived(cc_handle* h, double* const* out);
/* Restart files of the Navier-Stokes handle (as cc_euler2d_checkpoint_*,
 * magic "CCNS2CK1"; load checks grid, domain and precision). */
int cc_ns2d_checkpoint_save(cc_handle* h, const char* path);
int cc_ns2d_checkpoint_load(cc_handle* h, const char* path);

/* ---- spectral gravity without device allocation ----
 * No counterpart in the reference: an addition for callers that cannot call
 * cudaMalloc -- a host application whose memory manager owns the GPU's
 * memory, or a loop that must not pay cudaMalloc's implicit device
 * synchronisation.  Same result as cc_mhd2d_compute_gravity with
 * poisson_kind == CC_POISSON_FFT and precision == CC_FP64 (within 1e-12
 * relative, not bit for bit: the twiddle tables are built on the device),
 * computed from device arrays: rho (input) and gx, gy (outputs) are
 * caller-owned device pointers,
 * FP64, Nx*Ny each, q = j*Nx + i.  Work is queued on `stream`
 * (cudaStream_t, NULL = legacy default stream) and the call returns without
 * waiting for it.
 *
 * Scratch lives in one fixed device array inside the library (about 6.6 MB,
 * held by every GPU that loads the library until the process exits); nothing
 * is allocated or freed.  Limits: periodic, Nx and Ny powers of two with
 * 4 <= Nx, Ny <= CC_NOALLOC_MAX_SIDE and Nx*Ny <= CC_NOALLOC_MAX_CELLS;
 * larger grids return CC_ERR_TOO_LARGE.  Parameters asking for another solver
 * (poisson_kind other than CC_POISSON_FFT), FP32, or a non-periodic axis
 * return CC_ERR_UNSUPPORTED.
 * The first call on a device looks up the array's device address and raises
 * the FFT kernels' shared-memory limits; make that first call before any
 * stream capture.  Every call reuses the same array, which keeps the last
 * call's contents (each call overwrites everything it reads, nothing needs to
 * start at zero): calls that overlap on the GPU -- on two streams, from two
 * host threads -- race and must be serialised by the caller. */
#define CC_ERR_TOO_LARGE -7
#define CC_NOALLOC_MAX_CELLS (1 << 18)
#define CC_NOALLOC_MAX_SIDE 4096
int cc_mhd2d_gravity_fft_noalloc(const cc_mhd2d_params* p, const double* rho, double* gx, double* gy, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CC_STEP_H */
