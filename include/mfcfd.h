/*
 * mfcfd.h - C ABI of the B200 q-LSKUM implicit iteration.
 *
 * The reference (a serial Fortran 90 meshfree Euler solver) keeps its point
 * cloud in a module global (``type(points) :: point``, data_structure.f90:
 * 7-59) and calls argument-less routines on it.  The solver loop is
 *
 *     call generate_split_stencils()          q_lskum.f90:25
 *     call aliasing()                         q_lskum.f90:26
 *     do t = 1, max_iters
 *         call fpi_solver(t)                  q_lskum.f90:29
 *     enddo
 *
 * This header is the drop-in boundary for that loop: the Fortran host keeps
 * its arrays and passes them by pointer; the library copies them to the GPU
 * once, keeps all iteration state resident there, and replaces each
 * ``call fpi_solver(t)`` with ``mfcfd_fpi_step(h, t, &res_new, &residue)``.
 *
 * Conventions
 *   - Arrays use the reference's Fortran layout: an array declared
 *     ``A(m, N)`` is passed as m*N contiguous values with the m entries of a
 *     point adjacent (column-major).  ``conn`` holds 1-based point indices.
 *   - Every entry point returns an int status (MFCFD_OK = 0).  No exception,
 *     exit, trap or abort crosses the boundary; ``mfcfd_last_error`` gives a
 *     message for the last failure on a handle.
 *   - A handle is not thread safe; separate handles may be used from
 *     separate host threads.  Each handle owns one CUDA stream.
 */
#ifndef MFCFD_H
#define MFCFD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define MFCFD_OK               0
#define MFCFD_ERR_ARG          1   /* bad argument (null pointer, size, index) */
#define MFCFD_ERR_CUDA         2   /* CUDA runtime failure */
#define MFCFD_ERR_STENCIL      3   /* a stencil exceeds the supported width */
#define MFCFD_ERR_SINGULAR     4   /* a least-squares determinant is zero */
#define MFCFD_ERR_NONFINITE    5   /* the density residual is not finite */
#define MFCFD_ERR_UNSUPPORTED  6   /* input the library does not handle */
#define MFCFD_ERR_NOMEM        7   /* device or host memory, or a host thread, could not be had */
#define MFCFD_ERR_TIMEOUT      8   /* a bounded device wait ran out */
#define MFCFD_ERR_IO           9   /* a file could not be read, parsed or written */
#define MFCFD_ERR_BUSY        10   /* a served request did not finish within the wait */

/* fields for mfcfd_get (Fortran layout, width x N) */
#define MFCFD_FIELD_PRIM      0    /* point%prim(5,N)        width 5  */
#define MFCFD_FIELD_U         1    /* point%U(5,N)           width 5  */
#define MFCFD_FIELD_Q         2    /* point%q(5,N)           width 5  */
#define MFCFD_FIELD_QM        3    /* point%qm(2,5,N)        width 10 */
#define MFCFD_FIELD_DQ        4    /* point%dq(3,5,N)        width 15 */
#define MFCFD_FIELD_DELT      5    /* point%delt(N)          width 1  */
#define MFCFD_FIELD_FLUX_RES  6    /* point%flux_res(5,N)    width 5  */
#define MFCFD_FIELD_DELUP     7    /* point%delUp(5,N)       width 5  */
#define MFCFD_FIELD_DELUN     8    /* point%delUn(5,N)       width 5  */
#define MFCFD_FIELD_DINV      9    /* D_inv of the last sweep, width 1 */

#define MFCFD_PRECISION_FP64  0    /* all FP64, bit-matched to the CPU oracle */
#define MFCFD_PRECISION_MIXED 1    /* flux reconstruction, limiter and the flux
                                      evaluations of both sweeps in FP32; the
                                      least-squares moments and 3x3 solves,
                                      D_inv, the increments, the state update,
                                      residual norms and forces in FP64.
                                      Requires MFCFD_SWEEP_CHAINS.  The FP32
                                      flux residual leaves a noise floor near a
                                      1e-5 drop of the density residual. */
#define MFCFD_PRECISION_MIXED_DC 2 /* defect correction: the flux residual (the
                                      right-hand side) in FP64 as in the plain
                                      path, the implicit LU-SGS operator (the
                                      sweeps' flux evaluations, and the fluxes of
                                      the state they difference against) in
                                      FP32, each sweep list's 3x3 solve folded
                                      into its terms' weights.  The iteration's
                                      fixed point is the FP64 one; below about a
                                      1e-5 drop it slows, since FP32 increments
                                      resolve the state only to FP32 (finish in
                                      FP64: mfcfd_set_precision).  Requires
                                      MFCFD_SWEEP_CHAINS. */

/*
 * Run-time form of the reference's compile-time constants (parameter.f90:
 * 8-33).  mfcfd_params_init fills the reference's values for a given Mach
 * number and angle of attack.
 */
typedef struct mfcfd_params {
    double power;             /* least-squares weight exponent (parameter.f90:21) */
    double vl_const;          /* Venkatakrishnan limiter K (parameter.f90:22) */
    double cfl;               /* CFL number (parameter.f90:23) */
    double rho_inf, u1_inf, u2_inf, u3_inf, pr_inf;   /* freestream (parameter.f90:29-33) */
    int32_t inner_iterations; /* second-order q-derivative passes (parameter.f90:24) */
    int32_t split_capacity;   /* split-list capacity: 22 reproduces the reference's
                                 storage (data_structure.f90:83-88) including
                                 overflow into the next point's column; 0 means
                                 unlimited lists */
    int32_t precision;        /* MFCFD_PRECISION_FP64 (default) or _MIXED */
    int32_t device;           /* CUDA device ordinal; -1 builds a host-only handle
                                 (stencils, alias, schedule) without device state */
    int32_t sweep_mode;       /* MFCFD_SWEEP_CHAINS (default), _DATAFLOW or _LEVELS */
    int32_t update_variant;   /* MFCFD_UPDATE_IMPLICIT (default) or MFCFD_UPDATE_EXPLICIT */
    int32_t sweep_variant;    /* MFCFD_SWEEPS_ALIAS (default) or MFCFD_SWEEPS_BACKUP */
    int32_t chain_warps;      /* CHAINS: warps of the schedule; 0 picks about twice the
                                 widest level (fewer warps leave SMs to other clouds) */
    int32_t gpu_setup;        /* 1: the set-up runs on params->device with the host's
                                 results.  mfcfd_create computes every topology array on
                                 the device (the host classifies and orders the points
                                 and assigns the chain warps) for the alias sweep driver,
                                 power 0 and no supersonic points;
                                 otherwise, and in mfcfd_prepare, the split stencils, alias
                                 search and sweep levels run on the device for the host's
                                 set-up */
    int32_t graphs;           /* chunks of iterations captured once as CUDA graphs and
                                 replayed: 1 (default) in mfcfd_run_batch, 2 also in
                                 single-handle runs, 0 never (kernels one by one) */
    int32_t chain_spread;     /* CHAINS: 1 runs the sweep as 4-warp blocks of which each SM
                                 holds one, so every warp has an SM sub-partition to
                                 itself; 0 (default) packs blocks as residency allows */
    int32_t storage_order;    /* MFCFD_ORDER_MORTON (default) or MFCFD_ORDER_INDEX */
    int32_t flux_blocks_per_sm;   /* CHAINS: the flux residual beside the forward sweep as a
                                     grid of this many blocks per SM walking the sweep's
                                     order; 0 (default): one block per four points */
} mfcfd_params;

/* Order of the points in device memory.  The set-up (split lists, alias
 * search, sweep order) always works on the reference's point indices, and
 * every array crossing this interface is in that index order; only the
 * device layout changes.  MORTON stores the points along a Morton (Z-order)
 * curve of their coordinates, so a point's neighbours lie near it in memory;
 * INDEX keeps the caller's order.  Results are the same bits either way. */
#define MFCFD_ORDER_INDEX     0
#define MFCFD_ORDER_MORTON    1

/* The reference ships two drivers of its sweep module.  ALIAS:
 * implicit_forward_and_reverse_sweeps.f90 (the active build) sweeps wall and
 * interior points in alias order.  BACKUP:
 * implicit_forward_and_reverse_sweeps_backup.f90 sweeps the point classes in
 * turn (wall, interior, outer with their own D_inv and L/U routines, then
 * supersonic copies), each in index order and reversed for the backward
 * sweep; a neighbour not yet updated in that order contributes its
 * increment from before the sweep. */
#define MFCFD_SWEEPS_ALIAS    0
#define MFCFD_SWEEPS_BACKUP   1

/* The reference ships two sources of its state_update module; a build
 * compiles one.  IMPLICIT: state_update_implicit.f90 (the active build).
 * EXPLICIT: state_update.f90 -- wall normal momentum set to zero, outer
 * points updated explicitly (Ubar - delt * flux_res), supersonic points
 * copying their nearest neighbour of any status. */
#define MFCFD_UPDATE_IMPLICIT 0
#define MFCFD_UPDATE_EXPLICIT 1

/* LU-SGS sweep schedules.  All give the reference's sequential result bit
 * for bit.  DATAFLOW: warps on all SMs take points in topological order and
 * poll (bounded) for the increments of the neighbours they read.  LEVELS: one
 * CTA processes level after level with a block barrier between levels. */
#define MFCFD_SWEEP_DATAFLOW  0
#define MFCFD_SWEEP_LEVELS    1
/* CHAINS: points are assigned to warps ahead of time so that a point usually
 * runs on the warp that processed its deepest dependency, which hands its
 * increment over in shared memory; other neighbours are polled for.  One
 * cooperative launch keeps all warps resident. */
#define MFCFD_SWEEP_CHAINS    2

typedef struct mfcfd_info {
    int32_t n_points;
    int32_t n_wall, n_outer, n_interior, n_supersonic;
    int32_t n_levels_forward;     /* depth of the forward-sweep schedule */
    int32_t n_levels_backward;
    int32_t max_level_width;
    int32_t split_overflows;      /* list entries written past split_capacity */
    int32_t shared_frame;         /* 1 if interior points share one frame */
    int64_t device_bytes;         /* device memory held by the handle */
    int32_t sweep_mode;           /* MFCFD_SWEEP_* of the handle */
    int32_t chain_warps;          /* CHAINS: warps of the schedule, else 0 */
    /* CHAINS: sweep terms (both directions) of shared-frame consumers whose
     * producer is a swept point, by where the increment is read: the warp's
     * shared-memory ring, global memory written by the same warp, or global
     * memory written by another warp */
    int64_t chain_terms_ring, chain_terms_local, chain_terms_cross;
    /* CHAINS: slots (sixths of an SM) the handle's chain sweep holds while it
     * runs (a 4-warp block 2 in mixed precision, 3 in FP64; an 8-warp block
     * 6), and the slots all chain sweeps running at once may hold on the
     * device (mfcfd_launch) */
    int32_t chain_slots, chain_slot_capacity;
    /* CHAINS: swept points outside the shared frame (walls) whose neighbour
     * fluxes at the start of the sweeps one extra kernel per iteration
     * computes for both sweeps; 0 when there are none or too many */
    int32_t g0_points;
    /* CHAINS: warps per block of the chain sweep (4 or 8); handles of one
     * mfcfd_run_group share it */
    int32_t chain_warps_per_block;
} mfcfd_info;

typedef struct mfcfd_handle mfcfd_handle;

/* Fill *p with parameter.f90's values: power 0, K 2, CFL 5, no inner
 * iterations, rho 1, u = Mach (cos a, sin a, 0), p = 1/1.4, capacity 22;
 * and the library's defaults: FP64, device 0, the chain schedule, graphs in
 * batches, the Morton storage order. */
void mfcfd_params_init(mfcfd_params *p, double mach, double aoa_deg);

/*
 * Build the split stencils (generate_connectivity.f90:12-246) and the sweep
 * order (implicit_aliasing.f90:13-44), validate them, and upload the cloud.
 * Replaces allocate_size + read_input_point_data + generate_split_stencils +
 * aliasing (data_structure.f90:63-104, point_preprocessor.f90:30-95,
 * q_lskum.f90:25-26).  tan1/tan2/nor are (3,N); conn is (27,N), 1-based.
 * On failure *out may still receive a handle that carries the message for
 * mfcfd_last_error; destroy it with mfcfd_destroy.
 */
int mfcfd_create(const mfcfd_params *params, int32_t n, const int32_t *status,
                 const double *x, const double *y, const double *z,
                 const double *tan1, const double *tan2, const double *nor,
                 const int32_t *nbhs, const int32_t *conn, const double *min_dist,
                 mfcfd_handle **out);

/*
 * mfcfd_create in two steps, for a host that prepares clouds while others
 * iterate (the request server below).  mfcfd_prepare does the host set-up
 * (stencils, alias, levels, the chain schedule for params->device, which
 * must be >= 0) and keeps host copies; mfcfd_device_bytes gives the device
 * memory that mfcfd_attach will allocate (or holds, once attached);
 * mfcfd_attach allocates and uploads.  Until attached, only the set-up
 * queries (stencils, alias, levels, info) and mfcfd_destroy apply.
 */
int mfcfd_prepare(const mfcfd_params *params, int32_t n, const int32_t *status,
                  const double *x, const double *y, const double *z,
                  const double *tan1, const double *tan2, const double *nor,
                  const int32_t *nbhs, const int32_t *conn, const double *min_dist,
                  mfcfd_handle **out);
int mfcfd_device_bytes(mfcfd_handle *h, int64_t *bytes);
int mfcfd_attach(mfcfd_handle *h);

/* Set point%prim (5,N) and zero delUp/delUn: initial_conditions.f90:18-29. */
int mfcfd_set_prim(mfcfd_handle *h, const double *prim);

/* One call of fpi_solver(t) (fpi_solver.f90:20-45): the seven phases on the
 * GPU; returns res_new (state_update_implicit.f90:187) and residue
 * (fpi_solver.f90:38-43).  Either output pointer may be NULL. */
int mfcfd_fpi_step(mfcfd_handle *h, int32_t t, double *res_new, double *residue);

/*
 * mfcfd_run in two halves, for a host that keeps several handles busy
 * (the request server): mfcfd_launch queues iterations t0 .. t0+iters-1
 * (1 <= iters <= 1024) on the handle's stream and returns; mfcfd_complete
 * then reports whether they have finished (*done), or waits for them with
 * wait != 0, and on completion fills res_hist (2*iters, may be NULL) as
 * mfcfd_run does.  One launch may be pending per handle.  Chain sweeps of
 * handles running at once must fit the device together: the launches'
 * mfcfd_info.chain_slots may add up to chain_slot_capacity at most.
 */
int mfcfd_launch(mfcfd_handle *h, int32_t t0, int32_t iters);
int mfcfd_complete(mfcfd_handle *h, int32_t wait, double *res_hist, int32_t *done);

/* The q_lskum loop (q_lskum.f90:28-32) for t = t0 .. t0+iters-1 without host
 * round trips; res_hist (2*iters, may be NULL) receives (res_new, residue)
 * per iteration. */
int mfcfd_run(mfcfd_handle *h, int32_t t0, int32_t iters, double *res_hist);

/*
 * Batches: iterations t0[i] .. t0[i]+iters-1 of `count` handles of one device
 * (each handle once), run concurrently -- every iteration of each handle is
 * launched in turn on the handles' own streams, so one cloud's
 * latency-bound sweeps overlap another's.  Handles whose chain-schedule
 * sweeps would not all be resident together run in successive waves.
 * res_hist (may be NULL) is count x iters x (res_new, residue); status (may
 * be NULL) gets each handle's result; the return value is the first error.
 */
int mfcfd_run_batch(mfcfd_handle *const *hs, int32_t count, const int32_t *t0, int32_t iters,
                    double *res_hist, int32_t *status);

/*
 * Groups (the q_lskum loop, q_lskum.f90:28-32, of several clouds at once; no
 * counterpart in the reference): iterations t0[i] .. t0[i]+iters-1 of up to
 * MFCFD_GROUP_MAX_CLOUDS handles of one device in lockstep, each sweep
 * direction of every handle in ONE kernel launch (the persistent multi-cloud
 * chain sweep); the other kernels of an iteration run per handle, on the
 * handles' own streams, between the group's sweeps.  The handles use the
 * chain schedule with the same block shape (mfcfd_info.chain_warps_per_block),
 * chain_spread and precision class (FP64, or MIXED / MIXED_DC), and their
 * mfcfd_info.chain_slots add up to chain_slot_capacity at most; otherwise
 * MFCFD_ERR_UNSUPPORTED, before anything runs.  Every handle gets the bits
 * mfcfd_run gives it.  A group waits each iteration for its slowest sweep,
 * so handles of similar size group best.  res_hist and status as in
 * mfcfd_run_batch.  Calls on disjoint handles may run from separate host
 * threads at once; as with mfcfd_launch, the chain sweeps running at the
 * same time must then fit the device together (their chain_slots add up to
 * chain_slot_capacity at most), or their bounded waits may run out
 * (MFCFD_ERR_TIMEOUT).
 */
#define MFCFD_GROUP_MAX_CLOUDS 32
int mfcfd_run_group(mfcfd_handle *const *hs, int32_t count, const int32_t *t0, int32_t iters,
                    double *res_hist, int32_t *status);

/* Copy a field to host memory (see MFCFD_FIELD_*). */
int mfcfd_get(mfcfd_handle *h, int32_t field, double *out);

/* Checkpoint / resume: the whole iteration state is prim (5,N) plus
 * delUn (5,N) (delUp equals delUn between iterations) and the residual
 * reference res_old.  set_state does not zero the increments. */
int mfcfd_get_state(mfcfd_handle *h, double *prim, double *delu, double *res_old);
int mfcfd_set_state(mfcfd_handle *h, const double *prim, const double *delu, double res_old);

/* The six split lists as the flux routines read them (xpos, xneg, ypos,
 * yneg, zpos, zneg): counts (6,N) and the first `width` entries of each
 * list (width,6,N), 1-based, 0 past the count. */
int mfcfd_get_stencils(mfcfd_handle *h, int32_t *counts, int32_t *lists, int32_t width);

/* point%alias(N) and point%point_with_alias(N) (implicit_aliasing.f90). */
int mfcfd_get_alias(mfcfd_handle *h, int32_t *alias, int32_t *point_with_alias);

/* Level of every point in the forward (dir 0) or backward (dir 1) sweep
 * schedule; -1 for points the sweeps skip. */
int mfcfd_get_levels(mfcfd_handle *h, int32_t dir, int32_t *level);

/* Connectivity of a cloud that has none: the k (<= 27) nearest neighbours
 * of every point, as the reference's input file carries them
 * (point_preprocessor.f90:30-35): conn (27,N) 1-based in increasing order of
 * (d2, j), d2 = dx*dx + dy*dy + dz*dz with dx = x(j) - x(i), zero padded;
 * nbhs(i) = k; min_dist(i) = sqrt(d2) of the nearest.  device >= 0 runs on
 * that GPU, device < 0 on the host's threads; both give the same arrays.
 * Coinciding points or n <= k give MFCFD_ERR_ARG (message in
 * mfcfd_last_error(NULL)). */
int mfcfd_knn(int32_t device, int32_t n, const double *x, const double *y, const double *z, int32_t k,
              int32_t *nbhs, int32_t *conn, double *min_dist);

/* Diagnostics: a 64-bit FNV-1a digest of one device array of the handle's
 * topology, by its DevCloud name ("geo", "fwd_ent", "ch_items0", ...), and its
 * size in bytes (-1: not allocated).  Two handles of one cloud and
 * parameters give equal digests whether their set-up ran on the host or on
 * the device. */
int mfcfd_debug_digest(mfcfd_handle *h, const char *name, uint64_t *digest, int64_t *bytes);

int mfcfd_get_info(mfcfd_handle *h, mfcfd_info *info);

/* The CUDA stream (cudaStream_t) all of the handle's work runs on, so a
 * caller can order its own work or timing events after it. */
int mfcfd_get_stream(mfcfd_handle *h, void **stream);

/* Phase timing.  While enabled, every iteration records CUDA events between
 * its phases; mfcfd_get_phase_times returns the summed device milliseconds
 * per phase (MFCFD_NPHASE entries, order below) and the iteration count
 * since profiling was enabled. */
#define MFCFD_NPHASE 7   /* q-derivatives, flux residual, D_inv, forward sweep,
                            backward sweep, state update, residual sum */
int mfcfd_set_profiling(mfcfd_handle *h, int32_t on);
int mfcfd_get_phase_times(mfcfd_handle *h, double *ms, int64_t *iters);

/*
 * Allocation-free recomputation of the last iteration's density residual.
 * (No counterpart in the reference; it exists for callers that must not
 * allocate device memory.)
 *
 * Some callers cannot call cudaMalloc at the point where they need a result:
 * a host whose device memory is owned by another allocator or memory pool,
 * or code that runs while allocation is forbidden.  This entry point
 * recomputes res_new of the most recent mfcfd_fpi_step / mfcfd_run
 * iteration from the handle's per-point residual terms, with the same
 * two-pass reduction, and allocates nothing: its scratch (one partial sum per
 * reduction block) is a fixed device array inside the library that every GPU
 * loading the library holds until the process exits.
 *
 * Limit: at most MFCFD_NOALLOC_MAX_TERMS residual terms (wall plus interior
 * points); larger clouds get MFCFD_ERR_UNSUPPORTED.  Before the first
 * completed iteration, after mfcfd_set_prim or mfcfd_set_state, and after an
 * iteration that returned MFCFD_ERR_TIMEOUT there is no valid residual, and
 * the call returns MFCFD_ERR_ARG.  The first call on a device looks up the
 * scratch array's device address.  The call is synchronous: it ends with a
 * device-to-host copy and a wait on the handle's stream, so it must never be
 * made while the handle's stream, or a stream joined to it, is being
 * captured.  All calls share the one array and it keeps the last call's
 * contents (every call overwrites all of it that it reads), so calls that
 * overlap on the GPU race: do not run two at once, on any stream.
 */
#define MFCFD_NOALLOC_MAX_TERMS (1024 * 4096)
int mfcfd_residual_noalloc(mfcfd_handle *h, double *res_new);

/*
 * Switch a handle between MFCFD_PRECISION_FP64 and MFCFD_PRECISION_MIXED_DC
 * between iterations (no counterpart in the reference).  The defect-
 * correction form converges like FP64 down to about a 1e-5 drop of the
 * density residual and then slows, because its FP32 sweeps resolve
 * increments only to FP32; switching to FP64 for the last part of a solve
 * (a "polish") reaches a 1e-6 drop in FP64's iteration count.  The state
 * and the residual reference carry over.  A MIXED_DC handle sweeps with
 * each list's 3x3 solve folded into its terms' weights and keeps the
 * unfolded weights (24 bytes per sweep term), which the switch to FP64 puts
 * back bit for bit.  Handles created MIXED (folded weights only) cannot
 * switch.
 */
int mfcfd_set_precision(mfcfd_handle *h, int32_t precision);

/*
 * Failure-detection test hook (no counterpart in the reference, which has no
 * failure detection).  Every device wait of the sweeps is bounded: when one
 * runs out, the kernel sets an error word and returns, and the step reports
 * MFCFD_ERR_TIMEOUT with that iteration's results invalid.  This hook makes
 * that happen on purpose without faulting or hanging the GPU: from the next
 * iteration on, point `point` (1-based; 0 turns the hook off) publishes none
 * of its sweep increments, so the points that read them wait until their
 * bound runs out.  wait_limit > 0 sets that bound in poll rounds (0: the
 * default, about a second).  After MFCFD_ERR_TIMEOUT the handle stays
 * usable: turn the hook off and set the state again (mfcfd_set_prim or
 * mfcfd_set_state) before the next step.
 */
int mfcfd_set_fault_hook(mfcfd_handle *h, int32_t point, int32_t wait_limit);

/*
 * File formats of the reference program, for a host that replaces the whole
 * Fortran program (meshfree_solver.f90:20-37), not only its solver loop.
 * Input follows Fortran list-directed READ (one READ per record; blanks,
 * commas or line ends between values; r*value repeats; E or D exponents).
 * Output has the layout of gfortran's list-directed WRITE (17 significant
 * digits, so the values read back exactly).  Handle-less calls report
 * through mfcfd_last_error(NULL) (per host thread).
 */
/* Number of point records in a 3d_input_data file. */
int mfcfd_count_input_points(const char *path, int32_t *n);
/* read_input_point_data (point_preprocessor.f90:25-36): n records of
 * `idx status x y z tan1(3) tan2(3) nor(3) nbhs conn(1:nbhs) min_dist` into
 * arrays laid out as mfcfd_create takes them (conn (27,N) zero-padded). */
int mfcfd_read_input_point_data(const char *path, int32_t n, int32_t *status, double *x, double *y,
                                double *z, double *tan1, double *tan2, double *nor, int32_t *nbhs,
                                int32_t *conn, double *min_dist);
/* initial_conditions (initial_conditions.f90:18-29): stored-solution.dat,
 * `x y z rho u1 u2 u3 p` per point, into prim (5,N). */
int mfcfd_read_stored_solution(const char *path, int32_t n, double *prim);
/* print_primal_output (post_processor.f90:13-44): writes primal-solution.dat
 * (x y z prim), flux-residual.dat (k status flux_res), qderivatives.dat
 * (k status dq(3,1:5,k)) and an empty normals.dat into directory dir. */
int mfcfd_print_primal_output(mfcfd_handle *h, const char *dir);
/* residue.dat lines `t res_new residue` (q_lskum.f90:22,31) for
 * t = t0 .. t0+iters-1 from an mfcfd_run history; append != 0 appends. */
int mfcfd_write_residue(const char *path, int32_t t0, int32_t iters, const double *res_hist, int32_t append);

/*
 * Aerodynamic coefficients of the current state (no counterpart in the
 * reference, which prints no forces).  F = -sum over wall points of
 * (p_i - p_inf) A_i nor_i, with A_i = wall_area / (number of wall points)
 * unless per-point areas were set; CL = F.(-sin a, cos a, 0) / q and
 * CD = F.(cos a, sin a, 0) / q with q = rho_inf V^2 ref_area / 2 and the
 * angle a and speed V of (u1_inf, u2_inf).  force (3, may be NULL) receives F.
 * The wall sum runs on the GPU in a fixed order.
 */
int mfcfd_forces(mfcfd_handle *h, double wall_area, double ref_area, double *cl, double *cd, double *force);

/*
 * Autotuner of the chain schedule (no counterpart in the reference): times
 * `iters` iterations (after one untimed) of each candidate warp count from
 * the current state, restores that state after each, and keeps the
 * fastest schedule.  candidates NULL with count 0 tries 1.5, 2, 3 and 4
 * times the widest sweep level (the default schedule uses 2).  *chosen
 * receives the kept schedule's warps and ms (count or 4 entries, may be
 * NULL) each candidate's milliseconds per iteration.  The schedule orders
 * the work only: results are the same bits with any choice.
 */
int mfcfd_tune_chain(mfcfd_handle *h, const int32_t *candidates, int32_t count, int32_t iters, int32_t *chosen,
                     double *ms);
/* Rebuild the chain schedule for about `warps` warps (prepared or attached
 * handle); *actual (may be NULL) receives the schedule's warps.  In a batch,
 * fewer warps per cloud (about the widest level) let more clouds share the
 * device; alone, about twice the widest level is fastest. */
int mfcfd_set_chain_warps(mfcfd_handle *h, int32_t warps, int32_t *actual);
/* Per-point areas A_i (N values; only wall points' are read) for
 * mfcfd_forces; NULL returns to the uniform wall_area split. */
int mfcfd_set_wall_areas(mfcfd_handle *h, const double *area);

int mfcfd_destroy(mfcfd_handle *h);

/* Message of the last failure on h; with h = NULL, of the calling thread's
 * last failed handle-less call (file functions). */
const char *mfcfd_last_error(const mfcfd_handle *h);
const char *mfcfd_strerror(int code);

/*
 * Request server: steady-state solves (cloud, Mach, angle of attack) served
 * with continuous batching on one GPU (no counterpart in the reference,
 * whose program runs one solve).  Submitted requests are prepared on host
 * threads (mfcfd_prepare), admitted in the order they become ready while
 * their device memory fits the budget (and live < max_live), then iterate
 * side by side in chunks of `chunk` iterations, each launched as soon as
 * its chain sweep fits beside the running ones (mfcfd_launch).  When a
 * chunk completes, a request whose residue is <= its residue_target, or
 * that reached max_iters, or that failed, is retired: its CL/CD are
 * computed, its state copied out and its device memory freed for the next
 * admission; the others go on without waiting for each other.  A request's
 * iterations do not depend on the others in the mix: the same request
 * alone gives the same bits.
 */
typedef struct mfcfd_server mfcfd_server;

typedef struct mfcfd_server_config {
    int32_t device;           /* CUDA device ordinal */
    int32_t max_live;         /* requests iterating at once; 0: memory is the only limit */
    int32_t setup_threads;    /* host threads preparing submitted clouds (1..64) */
    int32_t chunk;            /* iterations per live request per round (1..1024) */
    int64_t hbm_budget;       /* device bytes the live requests may hold; 0: 90% of free memory */
    int32_t chain_percent;    /* chain schedule of each request: this percentage of its widest
                                 sweep level in warps (100 suits many requests at once);
                                 0: the request's own setting */
    int32_t device_setup;     /* 1: each request is set up on the device when it is admitted
                                 (mfcfd_create with gpu_setup = 1) instead of on the host
                                 when it arrives; admission reserves
                                 MFCFD_DEVICE_SETUP_BYTES_PER_POINT bytes per point and
                                 then holds the handle's own count (mfcfd_device_bytes) */
    int32_t reserved[6];
} mfcfd_server_config;

#define MFCFD_DEVICE_SETUP_BYTES_PER_POINT 6144

typedef struct mfcfd_request {
    mfcfd_params params;      /* flow, precision, schedule; device is the server's */
    int32_t n;                /* the cloud, as mfcfd_create takes it (copied at submit) */
    const int32_t *status;
    const double *x, *y, *z, *tan1, *tan2, *nor;
    const int32_t *nbhs, *conn;
    const double *min_dist;
    const double *prim;       /* (5,N) initial state; NULL: the freestream of params with
                                 the normal velocity removed at wall points */
    int32_t max_iters;        /* upper bound, rounded up to a multiple of chunk */
    double residue_target;    /* converged when residue <= this after a round */
    double wall_area, ref_area;   /* CL/CD at retirement when both are > 0 */
    double polish_residue;    /* MIXED_DC requests: switch to FP64 once the residue is at
                                 or below this after a round (mfcfd_set_precision);
                                 0: never */
} mfcfd_request;

typedef struct mfcfd_result {
    int64_t id;
    int32_t status;           /* MFCFD_OK or the code that retired the request */
    int32_t converged;        /* residue reached residue_target */
    int32_t iters;            /* iterations run */
    int32_t n;
    double res_new, residue;  /* after the last iteration */
    double cl, cd;            /* 0 unless areas were given */
    double t_submit, t_ready, t_admit, t_done;   /* seconds on the server's clock */
    int64_t device_bytes;
    double run_s;             /* seconds its chunks ran: launch to observed completion, summed */
} mfcfd_result;

typedef struct mfcfd_server_stats {
    int64_t submitted, completed, failed;
    int64_t preparing, waiting, live;      /* requests in each state now */
    int64_t bytes_live, peak_bytes_live, hbm_budget;
    int64_t rounds, iterations;            /* chunks completed; iterations summed over requests */
    int64_t peak_live;
    int64_t slot_capacity;                 /* chain-sweep slots of the device (0 before the first admission) */
    double busy_s;                         /* seconds with at least one chunk running */
    double slot_s;                         /* occupied slots integrated over time (slot-seconds) */
} mfcfd_server_stats;

int mfcfd_server_create(const mfcfd_server_config *cfg, mfcfd_server **out);
/* Copies the request's arrays; *id identifies it for mfcfd_server_wait. */
int mfcfd_server_submit(mfcfd_server *s, const mfcfd_request *req, int64_t *id);
/* Waits up to timeout_s (< 0: no limit) for request id to retire; fills
 * *res and, when prim is not NULL, the final (5,N) state, then forgets the
 * request.  MFCFD_ERR_BUSY if it has not retired within the wait. */
int mfcfd_server_wait(mfcfd_server *s, int64_t id, double timeout_s, mfcfd_result *res, double *prim);
int mfcfd_server_get_stats(mfcfd_server *s, mfcfd_server_stats *st);
/* Stops admitting, ends live requests after their current round (status
 * MFCFD_ERR_BUSY), and frees everything.  No other call on the server may be
 * in progress (a thread blocked in mfcfd_server_wait included) or follow. */
int mfcfd_server_destroy(mfcfd_server *s);

#ifdef __cplusplus
}
#endif

#endif /* MFCFD_H */
