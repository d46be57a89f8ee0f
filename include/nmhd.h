/* nmhd.h - C ABI of the B200-native ideal-MHD time step (libnmhd.so).
 *
 * Drop-in boundary for the reference's solver interface, class MHDSolver
 * (src/library/mhd_solver.hrb:150-276; generated src/library/mhd_solver.h:514-640).
 * Each entry point names the reference member it replaces.  Plain C types only:
 * sizes, pointers, status codes; no exceptions cross this boundary.
 *
 * Conventions
 *  - State is the reference's primitive state: 8 float32 fields of
 *    Sx*Sy*Sz values, x fastest, in the order of its .bin dump
 *    (density, vx, vy, vz, pressure, Bx, By, Bz).  B component d at index
 *    (x,y,z) is the field on the lower d-face of cell (x,y,z).
 *  - Sizes include margins (the reference's kSize{X,Y,Z}); every cell,
 *    margins included, is advanced, as in the reference.
 *  - The library owns device memory; the caller owns host buffers.
 *  - Calls are synchronous with respect to the host unless stated; a handle
 *    is not thread-safe.
 *  - Every call returns nmhd_status; nmhd_last_error() describes the last
 *    failure of a handle.
 */
#ifndef NMHD_H
#define NMHD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum nmhd_status {
  NMHD_OK = 0,
  NMHD_GOAL_REACHED = 1,        /* proceed(): goal time reached (reference returns true) */
  NMHD_TIMEOUT = 2,             /* proceed(): wallclock limit hit (reference returns false) */
  NMHD_STEP_LIMIT = 3,          /* proceed(): max_steps done before the goal */
  NMHD_ERR_INVALID_ARGUMENT = -1,
  NMHD_ERR_CUDA = -2,
  NMHD_ERR_IO = -3,             /* file cannot be opened, read or written */
  NMHD_ERR_SIZE_MISMATCH = -4,  /* .bin sizes differ from the solver's */
  NMHD_ERR_NUMERICAL = -5,      /* non-finite state, density <= 0 or pressure <= 0 */
  NMHD_ERR_OUT_OF_MEMORY = -6,
  NMHD_ERR_NOT_SUPPORTED = -7
} nmhd_status;

typedef enum nmhd_problem {
  NMHD_PROBLEM_NONE = 0,         /* no external acceleration */
  NMHD_PROBLEM_SHEARING_BOX = 1  /* Coriolis + tidal acceleration, shearing-periodic Y margins */
} nmhd_problem;

/* Options beyond the reference's scheme (nmhd_config.flags). */
typedef enum nmhd_flag {
  /* Refill the margins of the RK2 predictor from the interior before the
   * second stage (the Y shear fill with the displacement at t + dt/2, and the
   * Z copy).  The reference fills margins once per step and advances them
   * like the interior, so its second stage reads margin cells evolved in the
   * margin's own frame (from wrapped neighbours within two cells of the box
   * edge) and its interior depends on the margin width; with this flag the
   * interior results are the same, bitwise, for any margin width from 2, and
   * differ from the reference's scheme by truncation error.  Whole boxes
   * only (nmhd_proceed and the one-slab step); the batched, multi-slab and
   * adjoint paths return NMHD_ERR_NOT_SUPPORTED or reject the config. */
  NMHD_FLAG_HALO_PER_STAGE = 1,
  /* Face fluxes with fused multiply-adds, approximate division and square
   * root, and the HLLD solver's FP64 sub-expressions in float (kernel variant
   * 2 only; the update kernels stay exact).  Not bitwise: on noisy flows one
   * step from the same state is within 1e-5 of the reference's, relative to
   * each quantity's scale; on flows with exact symmetries, where the
   * reference's corner wind sums are exactly zero and CT takes the mean of
   * the two fluxes, rounding-size differences pick one of them and B
   * differs by up to ~1e-3 of its scale after one step.  The batched and
   * adjoint paths reject it. */
  NMHD_FLAG_FAST_ARITHMETIC = 2
} nmhd_flag;

/* Runtime form of the reference's compile-time simulation_config.h
 * (src/library/simulation_config_default.h, application overrides). */
typedef struct nmhd_config {
  int32_t size_x, size_y, size_z; /* kSize{X,Y,Z}: cells including margins */
  int32_t margin_y, margin_z;     /* kMarginSize{Y,Z}; X has no margin */
  float extent_x, extent_y, extent_z; /* kGlobalExtent{X,Y,Z} of the interior */
  float gamma;                    /* kGamma */
  float cfl;                      /* kCflFactor */
  int32_t problem;                /* nmhd_problem */
  float q, omega;                 /* kDifferentialRotationIndex, kOmega (shearing box) */
  int32_t space_order;            /* 2: minbee (reference default), 1: piecewise constant */
  int32_t time_order;             /* 2: midpoint RK2 (reference default), 1: Euler */
  int32_t flags;                  /* nmhd_flag bits, 0: the reference's scheme */
  /* kParallelSizeY: 0 or 1 for a whole box; P > 1 makes this solver one
   * radial slab of a box split over P ranks along Y (size_y counts the slab's
   * rows and margins, extent_y is the whole box's).  Its Y margins then come
   * from the neighbouring slabs through nmhd_halo_pack/nmhd_halo_unpack. */
  int32_t parallel_size_y;
} nmhd_config;

/* Conservation and field diagnostics, accumulated in FP64 over the interior
 * (monitor() of src/application/kepler_disk_demo/mhd_solver.curb:107-130 and
 * src/application/convergence_demo/mhd_solver.curb:61-100). */
typedef struct nmhd_diag {
  double mass;                   /* sum rho dV */
  double momentum[3];            /* sum rho v dV */
  double kinetic_energy;         /* sum rho v^2/2 dV */
  double internal_energy;        /* sum p/(gamma-1) dV */
  double magnetic_energy;        /* sum (face-averaged B^2)/2 dV */
  double total_energy;
  double bx2_mean, by2_mean;     /* <Bx^2>, <By^2> over all faces (reference monitor) */
  double maxwell_stress;         /* -<Bx By> with B at cell centres */
  double max_div_b;              /* max |div B| over interior cells */
  double volume;
} nmhd_diag;

typedef struct nmhd_solver nmhd_solver;

/* MHDSolver::MHDSolver(LocalSetup&) - allocates device state for `cfg`. */
nmhd_status nmhd_create(const nmhd_config *cfg, nmhd_solver **out);
/* ~MHDSolver */
void nmhd_destroy(nmhd_solver *s);

/* Replaces initialize_state()/set_initial_condition hooks: copy a primitive
 * state in.  fields[i] points to Sx*Sy*Sz floats, on the host
 * (on_device = 0) or on this solver's device (on_device = 1). */
nmhd_status nmhd_set_state(nmhd_solver *s, const float *const fields[8], int on_device);
/* Copy the primitive state out (the arrays MHDSolver::write dumps). */
nmhd_status nmhd_get_state(nmhd_solver *s, float *const fields[8], int on_device);

/* MHDSolver::read(std::string): sizes must match (else NMHD_ERR_SIZE_MISMATCH,
 * where the reference returns false). */
nmhd_status nmhd_read(nmhd_solver *s, const char *path);
/* MHDSolver::write(std::string): byte-identical to the reference's dump. */
nmhd_status nmhd_write(nmhd_solver *s, const char *path);

/* MHDSolver::proceed(goal_time, wallclock_time_limit)
 * (src/library/mhd_solver.inlrb:850-993).  Advances until current_time reaches
 * goal_time (rounded to float, as the reference's `Real goal_time`), the
 * wallclock limit in seconds passes (ignored if <= 0; checked between
 * batches of steps), or max_steps steps are done (ignored if <= 0).
 * Returns NMHD_GOAL_REACHED, NMHD_TIMEOUT, NMHD_STEP_LIMIT or an error;
 * *steps_done (may be NULL) receives the number of steps taken. */
nmhd_status nmhd_proceed(nmhd_solver *s, double goal_time, double wallclock_limit,
                         int64_t max_steps, int64_t *steps_done);
/* Builds, without running them, the CUDA graphs that nmhd_proceed(..., max_steps,
 * ...) launches (it steps in graphs of 16 steps and one of the remainder;
 * max_steps <= 0: the 16-step graph), so that a later proceed spends no host
 * time capturing them.  No counterpart in the reference, which launches every
 * kernel of every step from the host (mhd_solver.inlrb:850-993). */
nmhd_status nmhd_prepare(nmhd_solver *s, int64_t max_steps);

/* MHDSolver::current_time(), generation(), and the GlobalSetup fields that
 * load_state() restores. */
double nmhd_current_time(const nmhd_solver *s);
int64_t nmhd_generation(const nmhd_solver *s);
nmhd_status nmhd_set_time(nmhd_solver *s, double current_time, int64_t generation);

/* dt of the last `n` steps (most recent last); returns how many were stored.
 * The reference prints "t dt" to stderr every step (mhd_solver.inlrb:895). */
int64_t nmhd_dt_history(const nmhd_solver *s, float *out, int64_t n);

/* FP64 diagnostics of the current state (nmhd_diag). */
nmhd_status nmhd_diagnostics(nmhd_solver *s, nmhd_diag *out);

/* Device id of this solver, the CUDA stream its work runs on (a
 * cudaStream_t, may be set to the caller's stream), last error text. */
int nmhd_device(const nmhd_solver *s);
nmhd_status nmhd_set_stream(nmhd_solver *s, void *cuda_stream);
const char *nmhd_last_error(const nmhd_solver *s);

/* Per-kernel timing (no counterpart in the reference, which has no timers;
 * replaces its wallclock bench, src/application/optimize_mhd/main_detail.curb:27-57).
 * Runs `steps` steps launching every kernel separately with CUDA events around
 * it on the solver's stream; ms_out[i] receives the mean device time per step
 * of kernel class i and launches_out[i] (may be NULL) its kernel launches per
 * step.  Returns the
 * number of classes written (at most max), or a negative nmhd_status. */
int nmhd_profile(nmhd_solver *s, int steps, double *ms_out, double *launches_out, int max);
/* Kernel selection (the reference picks launch shapes with its Ruby autotuner,
 * src/application/optimize_mhd, kernel_call() in src/library/mhd_solver.inlrb:24-33).
 * variant 0: z-marching tiled kernels (32 x tile_rows cells per CTA,
 * tile_rows in {4, 8, 16}, z_chunk planes per CTA, 0 = whole height);
 * variant 1: per-cell flux and update kernels on 1-D blocks; variant 2:
 * per-cell kernels on 32x4x2 blocks; variant 3: the variant-2
 * kernels as a pipeline over chunks of z_chunk planes, so each chunk's face
 * fluxes are read back from L2 (nmhd_profile then times each whole stage as
 * its flux class); variant 4: the variant-2 flux kernel, then
 * constrained transport and the conserved update fused in one kernel per
 * stage (corner EMFs and new face B of a 32x4x2 tile in shared memory, its
 * inputs staged by tensor copies); variant 5 (the default): the variant-4
 * update after a flux kernel that first copies each 32x4x2 tile's stencil of
 * the stage input (all 8 fields, two cells around) into shared memory.  With
 * NMHD_FLAG_FAST_ARITHMETIC variants 2, 4 and 5 run the fast flux kernel
 * (5 is then 4) and the others are refused.  tile_rows is used
 * by variant 0 only, z_chunk by variants 0 and 3.  Every variant gives
 * bitwise identical results. */
nmhd_status nmhd_set_kernel(nmhd_solver *s, int variant, int tile_rows, int z_chunk);
/* The solver's kernel selection (any pointer may be NULL). */
nmhd_status nmhd_get_kernel(const nmhd_solver *s, int *variant, int *tile_rows, int *z_chunk);
/* Autotuner (replaces the reference's Ruby GA/parallel-tempering tuner of
 * launch dimensions, src/nushio_script/optimization.rb:33-140,
 * optimization_manager.rb:63-256).  Times `steps` steps of every kernel
 * variant and tile shape on this solver's box with CUDA events, starting each
 * trial from the current state, then restores the state and clock and selects
 * the fastest; solvers created later in the process for boxes of the same
 * shape, margins, problem and scheme start with that selection.  trials_out
 * (may be NULL) receives up to max_trials rows of
 * (variant, tile_rows, z_chunk, ms_per_step).  Returns the number of rows
 * written or a negative nmhd_status.  Every candidate gives bitwise the same
 * result, so tuning never changes the physics. */
int nmhd_autotune(nmhd_solver *s, int steps, double *trials_out, int max_trials);
/* Name of kernel class i of nmhd_profile (NULL when out of range). */
const char *nmhd_kernel_name(int i);

/* Allocation-free time stepping.  No counterpart in the reference (whose
 * MHDSolver owns Thrust vectors, src/library/mhd_solver.hrb:150-184).  For
 * callers that cannot allocate device memory: a host framework whose caching
 * allocator has reserved the device's memory, or a real-time loop where a
 * device allocation and the synchronisation it can bring are not allowed.
 * Advances a caller-owned box by up to nsteps steps (stopping at goal_time,
 * rounded to float) with the tiled kernels (kernel variant 0), which give
 * bitwise the same result as nmhd_proceed, keeping every intermediate in one
 * static device array of this library sized for NMHD_NOALLOC_MAX_CELLS cells
 * (about 28 MB, held by every GPU that loads the library until the process
 * exits).
 *   cfg        nmhd_create's rules, plus a whole box: parallel_size_y <= 1, flags 0
 *   state_in   device pointer, 8 x Sx*Sy*Sz floats (.bin field order); read only
 *   state_out  device pointer, same size, must not alias state_in; receives the result
 *   time, generation  in: the clock of state_in; out: the clock of the result
 * Boxes larger than NMHD_NOALLOC_MAX_CELLS are rejected with
 * NMHD_ERR_INVALID_ARGUMENT.  Calls no cudaMalloc/cudaFree.  The first call on
 * a device does the set-up: it looks up the array's device address with that
 * device current; make that first call before any stream capture.  All calls
 * share the array and it keeps the last call's contents: calls that overlap on
 * the GPU race.  Runs on
 * `cuda_stream` (NULL: the default stream), reads the control block back
 * every 16 steps (stopping once the goal is reached or the state is bad) and
 * returns when done.  A CUDA error pending from earlier work is reported as
 * NMHD_ERR_CUDA without launching anything.  Returns NMHD_GOAL_REACHED,
 * NMHD_STEP_LIMIT or an error; nmhd_noalloc_last_error() describes the last
 * error. */
#define NMHD_NOALLOC_MAX_CELLS 262144
nmhd_status nmhd_advance_noalloc(const nmhd_config *cfg, const float *state_in, float *state_out,
                                 double *time, int64_t *generation, double goal_time, int64_t nsteps,
                                 int64_t *steps_done, void *cuda_stream);
const char *nmhd_noalloc_last_error(void);

/* ---- Batched ensemble -------------------------------------------------------
 * Many independent boxes of uneven sizes (e.g. an ensemble over beta, shear
 * and seed) advanced together.  No counterpart in the reference, which runs
 * one compile-time box per process.  Every box has its own configuration,
 * state, clock and CFL time step (reduced per box), and is advanced bitwise as
 * nmhd_proceed would advance it alone.  Each kernel of a step is one launch
 * over all boxes (per group of 128 boxes, whose descriptors travel in the
 * launch's parameter block), either persistent (a resident grid walking tile
 * ranges) or one tile per CTA, as nmhd_batch_autotune picks; each box has its
 * own tile shape (nmhd_batch_tile_shape); batches of steps are one CUDA graph.
 * Batched boxes use time_order 2 and no Z margins. */
typedef struct nmhd_batch nmhd_batch;
nmhd_status nmhd_batch_create(const nmhd_config *boxes, int n, nmhd_batch **out);
void nmhd_batch_destroy(nmhd_batch *b);
int nmhd_batch_size(const nmhd_batch *b);
/* State of box `box`, as nmhd_set_state/nmhd_get_state. */
nmhd_status nmhd_batch_set_state(nmhd_batch *b, int box, const float *const fields[8], int on_device);
nmhd_status nmhd_batch_get_state(nmhd_batch *b, int box, float *const fields[8], int on_device);
/* Every box's state at once: fields holds 8 pointers per box, box after box
 * (8 * nmhd_batch_size pointers); one round trip to the boxes' control blocks
 * instead of one per box. */
nmhd_status nmhd_batch_set_states(nmhd_batch *b, const float *const *fields, int on_device);
nmhd_status nmhd_batch_get_states(nmhd_batch *b, float *const *fields, int on_device);
/* Clock of box `box` (current_time, generation). */
nmhd_status nmhd_batch_clock(nmhd_batch *b, int box, double *time, int64_t *generation);
/* Advances every box until all reach goal_time or max_steps steps are done
 * (semantics of nmhd_proceed, per box; a box that reached the goal waits).
 * *steps_done: steps taken by the box that took most. */
nmhd_status nmhd_batch_proceed(nmhd_batch *b, double goal_time, int64_t max_steps, int64_t *steps_done);
/* Builds, without running them, the CUDA graphs nmhd_batch_proceed(..., max_steps,
 * ...) launches (as nmhd_prepare). */
nmhd_status nmhd_batch_prepare(nmhd_batch *b, int64_t max_steps);
/* Stream of the batch's work, as nmhd_set_stream (NULL: a stream of its own). */
nmhd_status nmhd_batch_set_stream(nmhd_batch *b, void *cuda_stream);
/* Tile of box `box` in the batched kernels: tile_x x tile_y x tile_z cells (256
 * threads), chosen per box to launch the fewest padded cells, at least 8 wide
 * in x; ties keep 32 x 4 x 2. */
nmhd_status nmhd_batch_tile_shape(const nmhd_batch *b, int box, int *tile_x, int *tile_y, int *tile_z);
/* The same rule for a box configuration, without a batch (host only). */
nmhd_status nmhd_batch_tile_rule(const nmhd_config *box, int *tile_x, int *tile_y, int *tile_z);
/* Kernel launches of one batched time step with the current schedules. */
int nmhd_batch_launches_per_step(const nmhd_batch *b);
/* Schedule of stage kernel `kernel` (0 face fluxes, 1 constrained transport,
 * 2 conserved update): persistent = 1 for the resident grid walking tile
 * ranges, 0 for one tile per CTA (the default); split = 1 (the default) runs
 * the boxes with 32 x 4 x 2 tiles in a launch of their own through a kernel
 * compiled for that shape (fewer registers), 0 runs every box in one launch of
 * the general form (half the launches: better for many small boxes).
 * kernel = 3 is the fused pass: split = 1 runs constrained transport and the
 * conserved update of the 32 x 4 x 2 boxes as one kernel (the single-box fused
 * epilogue; it takes effect while kernels 1 and 2 are split), persistent its
 * schedule; split = 0 (the default) turns it off.  kernel = 4 is the staged
 * flux pass: split = 1 computes the face fluxes of the 32 x 4 x 2 boxes from a
 * shared-memory copy of each tile's stencil (the single-box variant-5 flux
 * kernel; it takes effect while kernel 0 is split), persistent its schedule. */
nmhd_status nmhd_batch_set_schedule(nmhd_batch *b, int kernel, int persistent, int split);
/* Schedule autotuner of the batch (the batched counterpart of nmhd_autotune).
 * Times `reps` launches of each stage kernel (face fluxes, constrained
 * transport, conserved update) in every schedule (persistent or not, split or
 * not) on the boxes' current states with CUDA events, keeps the fastest per
 * kernel, then times the face fluxes against the staged flux pass and the
 * stage update (kernels 1 and 2) against the fused pass, each one tile per
 * CTA and persistent, and keeps the fastest; states and clocks are left
 * unchanged.  trials_out (may be NULL) receives up to max_trials rows of
 * (kernel, persistent, split, ms per launch), the two comparisons as rows
 * (4, persistent, staged, ms per flux launch) and (3, persistent, fused, ms
 * per stage update).  Returns the number of rows written or a negative
 * nmhd_status.
 * Every schedule gives bitwise the same result. */
int nmhd_batch_autotune(nmhd_batch *b, int reps, double *trials_out, int max_trials);
const char *nmhd_batch_last_error(const nmhd_batch *b);

/* ---- Differentiation ---------------------------------------------------------
 * Gradients of a time-averaged diagnostic with respect to the initial state.
 * No counterpart in the reference.  The differentiated step is the solver's
 * own step with its time steps frozen (no derivative through the CFL dt) and
 * its non-smooth choices frozen at the branch taken: minbee limiter slopes,
 * the HLLD fan region, min/max of the wave speeds, sign(Bx) and the CT
 * upwind corner selection.  All runs start from the solver's current state
 * and clock and leave the solver's state, clock and time-step history
 * unchanged.  `dt_seq` (host, nsteps floats) freezes the time steps; NULL
 * means "the steps the CFL condition gives", i.e. exactly what nmhd_proceed
 * would take from this state.  `dt_out` (host, nsteps floats, may be NULL)
 * receives the time steps used.  At most NMHD_ADJOINT_MAX_STEPS steps. */
#define NMHD_ADJOINT_MAX_STEPS 4096
typedef enum nmhd_loss_kind {
  /* J = (1/nw) sum_{n = first_step}^{last_step} <-Bx By>_n: the Maxwell stress
   * of the state after n steps (n = 0: the initial state), averaged over the
   * interior cells with B at cell centres (nmhd_diag.maxwell_stress), and over
   * the nw = last_step - first_step + 1 states of the window. */
  NMHD_LOSS_MAXWELL_STRESS = 1
} nmhd_loss_kind;
typedef struct nmhd_loss_spec {
  int32_t kind;       /* nmhd_loss_kind */
  int32_t first_step; /* 0 <= first_step <= last_step <= nsteps */
  int32_t last_step;
  int32_t reserved;   /* 0 */
} nmhd_loss_spec;
/* FP32 forward run of nsteps steps with the production kernels; *loss_out
 * receives J. */
nmhd_status nmhd_loss_run(nmhd_solver *s, int32_t nsteps, const nmhd_loss_spec *loss, const float *dt_seq,
                          double *loss_out, float *dt_out);
/* FP32 adjoint: J and dJ/d(initial state) in grad[8] (8 fields of Sx*Sy*Sz
 * floats, host or device per on_device; margin entries that the first margin
 * fill overwrites get 0).  The forward run stores a checkpoint every
 * ckpt_every steps; the reverse sweep recomputes each segment from its
 * checkpoint, keeping that segment's stage inputs and fluxes, then runs the
 * hand-written adjoint kernels of every stage backwards. */
nmhd_status nmhd_adjoint_run(nmhd_solver *s, int32_t nsteps, int32_t ckpt_every, const nmhd_loss_spec *loss,
                             const float *dt_seq, double *loss_out, float *dt_out, float *const grad[8],
                             int on_device);
/* The same in FP64 (forward and adjoint in double from the float initial
 * state); dt_seq is required; grad on the host. */
nmhd_status nmhd_adjoint_run_f64(nmhd_solver *s, int32_t nsteps, int32_t ckpt_every,
                                 const nmhd_loss_spec *loss, const float *dt_seq, double *loss_out,
                                 double *const grad[8]);
/* FP64 tangent-linear run: J and its directional derivative dJ[dir] along
 * dir[8] (host, 8 fields of Sx*Sy*Sz doubles; NULL: J only), forward mode in
 * double.  The run starts from the solver's float state plus shift*dir, in
 * double, so central differences of J in FP64 can use perturbations far below
 * float rounding (shift is ignored when dir is NULL).  dt_seq is required. */
nmhd_status nmhd_tlm_run(nmhd_solver *s, int32_t nsteps, const nmhd_loss_spec *loss, const float *dt_seq,
                         const double *const dir[8], double shift, double *loss_out, double *dloss_out);
/* Memory for forward tapes beyond the last segment's.  The forward run of
 * nmhd_adjoint_run(_f64) stores a checkpoint every ckpt_every steps and keeps
 * the tapes of the last segments; the reverse sweep recomputes only the
 * segments whose tapes were not kept.  bytes = -1 (default): as many segments
 * as fit in half of the device memory free at the run; 0: the last segment
 * only (least memory); > 0: that many bytes for further segments.  The
 * gradient does not depend on it (bitwise).  When segments are recomputed, one
 * more segment's tape is held for the recomputation that overlaps the
 * reverse sweep.  nmhd_adjoint_kept_segments: how many segments the last
 * run's forward kept. */
nmhd_status nmhd_adjoint_set_tape_budget(nmhd_solver *s, int64_t bytes);
int32_t nmhd_adjoint_kept_segments(const nmhd_solver *s);
/* Device time of the last nmhd_adjoint_run / nmhd_adjoint_run_f64 in ms:
 * [0] forward run with checkpoints, [1] segment recomputation (on a stream of
 * its own, overlapping [2]: the recomputation of a segment runs beside the
 * adjoint of the segment after it, in a second tape slot), [2] the reverse
 * sweep (adjoint kernels, waiting for recomputed segments), [3] the whole
 * run, [0] + [2]. */
nmhd_status nmhd_adjoint_timing(const nmhd_solver *s, double ms_out[4]);

/* ---- Radial slab decomposition (kParallelSizeY = P ranks along Y) ----
 * Replaces the reference's host-staged MPI halo exchange, MHDSolver::
 * communicate (src/library/mhd_solver.inlrb:283-493), and the dt reduction of
 * proceed (:870-893, MPI_Allreduce MIN), for a solver created with
 * parallel_size_y = P: one step of rank r is
 *   nmhd_halo_pack(s, send_inc, send_dec)   gather the shear-shifted boundary rows
 *   transport: send_inc to rank (r+1)%P and send_dec to rank (r-1+P)%P;
 *              receive recv_inc from (r-1+P)%P and recv_dec from (r+1)%P
 *   nmhd_halo_unpack(s, recv_inc, recv_dec) fill the Y (and Z) margins, CFL time of the slab
 *   reduce:    the float at nmhd_cfl_slot(s) := its minimum over the P ranks
 *   nmhd_step_stages(s)                     the RK stages with the common dt
 * These enqueue on the solver's stream and return at once; the caller's
 * transport (NCCL send/recv and all-reduce on the same stream, or device
 * copies between slabs of one process) runs between them.  Halo buffers are
 * device memory of nmhd_halo_count(s) floats (8 fields x Sx x margin_y x Sz,
 * the reference's mpi_buffer_y_* layout).  With P = 1 and each message
 * delivered to itself this is exactly nmhd_proceed's step.
 * nmhd_slab_begin prepares a run toward goal_time (proceed()'s goal);
 * nmhd_slab_poll waits for the stream and returns NMHD_GOAL_REACHED once the
 * goal step is done, NMHD_ERR_NUMERICAL on a bad state, else NMHD_OK; steps
 * after the goal step are no-ops.  nmhd_proceed, nmhd_profile and
 * nmhd_autotune refuse a slab (P > 1) with NMHD_ERR_NOT_SUPPORTED. */
int64_t nmhd_halo_count(const nmhd_solver *s);
nmhd_status nmhd_slab_begin(nmhd_solver *s, double goal_time);
nmhd_status nmhd_halo_pack(nmhd_solver *s, float *send_inc, float *send_dec);
nmhd_status nmhd_halo_unpack(nmhd_solver *s, const float *recv_inc, const float *recv_dec);
float *nmhd_cfl_slot(nmhd_solver *s);
/* The reduce step for n slabs of one process that share one device and one
 * stream (nmhd_set_stream): one kernel on that stream. */
nmhd_status nmhd_cfl_min(nmhd_solver *const *slabs, int n);
nmhd_status nmhd_step_stages(nmhd_solver *s);
nmhd_status nmhd_slab_poll(nmhd_solver *s, int64_t *generation, double *time);

/* Library version string. */
const char *nmhd_version(void);

#ifdef __cplusplus
}
#endif
#endif /* NMHD_H */
