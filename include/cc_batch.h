/*
 * cc_batch.h -- batched ensemble of independent 2D resistive-MHD instances.
 *
 * No reference counterpart: the reference runs one grid per process
 * (mhd2d_resistive_hlld_ct_gravity.cpp main(), M2:1051-1123).  An ensemble
 * handle advances n instances of that solver, each with its own grid size,
 * domain, boundary kind, physics constants, t_end and CFL dt, through one
 * persistent stage kernel per RK stage over a work-list of tiles of all
 * instances; a run of steps is captured as one CUDA graph.
 *
 * Each instance's step is the single-grid step (cc_mhd2d_*, M2:838-869)
 * except for the Poisson solve: with gravity_on the instance must ask for
 * poisson_kind == CC_POISSON_DIRECT, the exact (to roundoff) solution of the
 * discrete Poisson problem the reference's SOR (M2:207-223) iterates towards:
 * same 5-point Laplacian, same clamp/wrap boundary rule, zero-mean potential.
 * Its density mean is reduced per instance in a fixed tile order, so an
 * instance's result does not depend on the rest of the batch.
 *
 * State arrays are the single-grid ones: f = {rho, mx, my, mz, E, Bz, Bx_f,
 * By_f} in the reference layouts (cc_step.h).  All instances share one
 * precision.  Statuses and cc_last_error / cc_destroy / cc_set_stream /
 * cc_get_perf are those of cc_step.h.
 */
#ifndef CC_BATCH_H
#define CC_BATCH_H

#include "cc_step.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Largest side of an instance with gravity (the x transform is a dense nx*nx basis). */
#define CC_BATCH_MAX_DIRECT_SIDE 2048

typedef struct cc_batch_info {
    int32_t n;               /* instances                                  */
    int32_t precision;       /* CC_FP64 or CC_FP32                         */
    int64_t cells;           /* sum of Nx*Ny over instances                */
    int32_t shape;           /* stage candidate in use                     */
    int32_t n_shapes;        /* candidates: tile shapes x {persistent, one CTA per tile} */
    int32_t tile_x, tile_y;  /* its tile                                   */
    int32_t stage_tiles;     /* work-list length of the stage kernel       */
    int32_t stage_ctas;      /* persistent CTAs of the stage kernel        */
    int32_t reduce_tiles;    /* 32x8 reduce tiles (one partial each)       */
    int32_t poisson_tiles;   /* GEMM tiles of the direct solve             */
    int64_t device_bytes;    /* device memory held by the handle           */
    int32_t poisson_tile;    /* their edge: 32 or 64 (CUDA cores), 128 (every solved instance on the
                                tcgen05 tensor cores: FP32 with Nx % 4 == 0), -128 (some of them) */
    int32_t reserved;
} cc_batch_info;

/* params: n instance descriptions (Nx, Ny >= 4; same precision). */
int cc_batch_create(const cc_mhd2d_params* params, int n, cc_handle** out);

/* f: 8 arrays of instance inst (reference layouts). */
int cc_batch_upload(cc_handle* h, int inst, const double* const* f);
int cc_batch_download(cc_handle* h, int inst, double* const* f);

/* dt of every instance from its resident state (compute_dt, M2:579-598); dt: n entries. */
int cc_batch_compute_dt(cc_handle* h, double* dt);

/* nsteps of the main() loop body (M2:1111-1117) for every instance, each with
 * its own dt clamped to its t_end; an instance with t >= t_end keeps its
 * state.  t: NULL (continue from the device clocks) or n entries, read as the
 * start times and overwritten with the end times. */
int cc_batch_advance(cc_handle* h, int nsteps, double* t);

int cc_batch_diagnostics(cc_handle* h, int inst, cc_diag* d);
/* Every instance's simulated time (n doubles, instance order): the clocks
 * cc_batch_advance keeps on the device, read with one copy. */
int cc_batch_times(cc_handle* h, double* t);

/* Time every stage candidate on the resident state (reps launches each) and
 * keep the fastest; shape / ms (may be NULL) receive the choice and its mean
 * stage time.  Candidate c uses tile shape c % S of the S compiled shapes,
 * launched persistent (c < S: one CTA per resident slot walking a contiguous
 * run of the tile work-list) or flat (c >= S: one CTA per tile). */
int cc_batch_autotune(cc_handle* h, int reps, int* shape, double* ms);
/* Use candidate `shape` (0 <= shape < n_shapes). */
int cc_batch_set_shape(cc_handle* h, int shape);
int cc_batch_get_info(cc_handle* h, cc_batch_info* info);

#ifdef __cplusplus
}
#endif

#endif /* CC_BATCH_H */
