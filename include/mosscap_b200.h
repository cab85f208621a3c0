/*
 * mosscap_b200 -- C ABI of the B200 (sm_100a) finite-volume Euler step.
 *
 * The library replaces the hydro hooks that Mosscap installs on its
 * Simulation aggregate (source/Simulation.hpp:38-62):
 *   Simulation::time_step   void(Simulation&, fp_t dt)   -> mc_time_step
 *   Simulation::compute_dt  f64(const Simulation&)       -> mc_compute_dt
 *   fill_bcs(const Simulation&)                          -> mc_fill_bcs
 * plus a device-resident driver of the main loop (source/main.cpp:54-72),
 * mc_advance, which keeps dt, the clock and the output clamp on the GPU.
 *
 * Data contract (source/State.hpp:101-152): the conserved state Q is a
 * caller-owned device array of doubles laid out [var][k][j][i] (i fastest)
 * with ng ghost cells on both ends of every active axis; the variables are
 * rho, m_x[, m_y[, m_z]], E followed by num_tracers passive mass densities.
 * Q enters every step with its ghost cells filled (as the reference's
 * time_step assumes) and leaves with them filled.
 *
 * Every call is exception-free and returns an mc_status. Calls are ordered
 * on the stream they are given (a cudaStream_t passed as void*; NULL is the
 * legacy default stream) and return without waiting, except where noted.
 * One context must not be used from two threads at once.
 */
#ifndef MOSSCAP_B200_H
#define MOSSCAP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MC_ABI_VERSION 1

typedef enum {
    MC_OK = 0,
    MC_ERR_INVALID_ARGUMENT = 1, /* bad descriptor, null pointer, size out of range */
    MC_ERR_UNSUPPORTED = 2,      /* combination the library does not implement */
    MC_ERR_CUDA = 3,             /* a CUDA runtime call failed; see mc_last_error */
    MC_ERR_OUT_OF_MEMORY = 4,
    MC_ERR_STATE = 5             /* the device status word holds a physics flag */
} mc_status;

/* Physics flags accumulated on the device (mc_get_status). */
#define MC_FLAG_NONFINITE 0x1u     /* a non-finite value in a state the step read or wrote */
#define MC_FLAG_NEG_DENSITY 0x2u   /* rho <= 0 */
#define MC_FLAG_NEG_PRESSURE 0x4u  /* p <= 0 */
#define MC_FLAG_BAD_DT 0x8u        /* dt <= 0 or not finite */
#define MC_FLAG_EOS 0x10u          /* a non-ideal EOS update met a state the reference aborts on */
#define MC_FLAG_TIMEOUT 0x20u      /* a kernel's bounded wait (a TMA tile copy) gave up; the tile was not updated */

/* Enum values equal the reference's ordinals. */
typedef enum { /* source/Reconstruct.hpp:10-15 */
    MC_RECON_FOG = 0,
    MC_RECON_MUSCL = 1,
    MC_RECON_PPM = 2,
    MC_RECON_WENO5Z = 3
} mc_reconstruction;

typedef enum { /* source/Reconstruct.hpp:22-26 */
    MC_LIMITER_VANLEER = 0,
    MC_LIMITER_MONOTONIZED_CENTRAL = 1,
    MC_LIMITER_MINMOD = 2
} mc_slope_limiter;

typedef enum { /* source/Riemann.hpp:10-14 */
    MC_RIEMANN_RUSANOV = 0,
    MC_RIEMANN_HLL = 1,
    MC_RIEMANN_HLLC = 2
} mc_riemann_solver;

typedef enum { /* source/TimeStepping.hpp:10-14 */
    MC_STEPPER_RK2 = 0,
    MC_STEPPER_SSPRK3 = 1,
    MC_STEPPER_SSPRK4 = 2
} mc_time_stepper;

typedef enum { /* source/State.hpp:62-70 */
    MC_BC_WALL = 0,
    MC_BC_PERIODIC = 1,
    MC_BC_SYMMETRIC = 2,
    MC_BC_SYMMETRIC_OUTFLOW_DIODE = 3,
    MC_BC_ZEROGRAD = 4,
    MC_BC_CONSTANT = 5,
    MC_BC_USERFN = 6 /* ghost cells left to the caller's hook after each fill */
} mc_boundary_type;

typedef enum {
    /* Every operation in the reference's order without fused multiply-adds:
     * bit-identical to the reference's CPU build. */
    MC_PRECISION_FP64 = 0,
    /* Reconstruction, Riemann fluxes and their EOS calls in FP32; the
     * conserved state, the primitive recovery from it (pressure from total
     * energy), the flux-divergence accumulation and dt stay FP64. */
    MC_PRECISION_FP32_COMPENSATED = 1
} mc_precision;

/* Grid description; mirrors GridSize / State / Boundaries
 * (source/State.hpp:72-152, set up as in source/SetupModules.hpp:9-136). */
typedef struct {
    int32_t num_dim;      /* 1, 2 or 3 */
    int32_t xc, yc, zc;   /* cells per axis including ghosts; 1 on inactive axes */
    int32_t ng;           /* ghost cells per side on active axes */
    int32_t num_tracers;  /* passive scalars after the 2+num_dim hydro variables */
    double dx;            /* cell width, equal on every axis */
    double loc[3];        /* lower corner of the first interior cell (State::loc) */
    int32_t bc[6];        /* xs, xe, ys, ye, zs, ze (mc_boundary_type) */
    double bc_const[6][5];/* conserved values for MC_BC_CONSTANT faces, in variable order */
} mc_grid;

/* Numerical scheme; mirrors NumericalSchemes + Eos + max_cfl
 * (source/Simulation.hpp:17-22, source/Eos.hpp:27-42). */
typedef struct {
    int32_t reconstruction; /* mc_reconstruction */
    int32_t slope_limiter;  /* mc_slope_limiter (ignored by FOG and WENO5-Z) */
    int32_t riemann_solver; /* mc_riemann_solver */
    int32_t time_stepper;   /* mc_time_stepper */
    int32_t precision;      /* mc_precision */
    double gamma;           /* ideal-gas ratio of specific heats */
    double max_cfl;         /* dt = max_cfl * min over cells of dx / (c_s + |v|) */
} mc_scheme;

/* Time bookkeeping of Simulation / OutputConfig (source/Simulation.hpp:40-44,
 * source/Output.hpp:15-23): compute_dt clamps dt so that a step ends exactly
 * on min(max_time, prev_output_time + output_delta) (source/Hydro.cpp:231-241). */
typedef struct {
    double time;
    double max_time;
    double prev_output_time;
    double output_delta;
} mc_clock;

typedef struct mc_ctx mc_ctx;

/* Create a context for one grid + scheme on the current CUDA device.
 * Allocates the stage buffers (two states' worth) and a small device block.
 * Rejects ng below the reconstruction's need (FOG 1, MUSCL 2, PPM / WENO5-Z 3;
 * source/Reconstruct.hpp:47-61) and active axes with fewer than ng interior
 * cells. Replaces Simulation setup (source/SetupModules.hpp:9-168). */
mc_status mc_create(const mc_grid* grid, const mc_scheme* scheme, mc_ctx** out);
mc_status mc_destroy(mc_ctx* ctx);

/* Simulation::user_bc (source/Simulation.hpp:55, called at the end of
 * fill_bcs, source/Boundaries.hpp:146-148): a host function that enqueues on
 * `stream` the caller's own ghost fill of a state buffer. It is called after
 * mc_fill_bcs and after every stage, with the stage's output buffer (which
 * may be a library-owned buffer, not the caller's Q), and must be idempotent:
 * mc_advance may call it for steps the device has already skipped. Required
 * when any active face is MC_BC_USERFN. fn = NULL removes the hook. */
mc_status mc_set_user_bc(mc_ctx* ctx, void (*fn)(void* user, double* Q, void* stream), void* user);

/* Domain-wide CFL minimum for a grid split over ranks. compute_dt reduces
 * over the whole domain (source/Hydro.cpp:209-229); when each rank holds one
 * part, the ranks' minima must be combined before dt is formed. fn is a host
 * function that enqueues on `stream` that combination, in place, for the
 * device word `cfl_min_bits`: the bit pattern of the non-negative CFL
 * minimum, so a 64-bit integer MIN over the ranks is the minimum of the
 * values. The library calls it wherever it forms a dt: in mc_compute_dt,
 * and in mc_advance before every step's dt, so a device-driven loop needs no
 * host round trip per step. fn = NULL removes it. No counterpart in the
 * reference, which runs on one domain. */
mc_status mc_set_cfl_reduce_hook(mc_ctx* ctx, void (*fn)(void* user, uint64_t* cfl_min_bits, void* stream),
                                 void* user);

/* Slab decomposition over ranks (one GPU per rank). The problem is split
 * along its slowest active axis (y in 2D, z in 3D) into one slab per rank;
 * each rank creates its context for its own slab (its interior cells along
 * that axis, with ghost layers, the global problem's face kinds) and then
 * joins the decomposition with the id rank 0 obtained from mc_slab_unique_id
 * and handed to every rank (through any host channel). From then on the
 * library itself fills the ghost layers between neighbouring slabs after
 * every stage and after mc_fill_bcs (NCCL send/receive of the bordering ng
 * layers, in the stream), and reduces the CFL minimum over all ranks
 * wherever it forms a dt (NCCL all-reduce MIN in the stream, exact because a
 * minimum does not depend on order): every rank takes the same dt and the
 * slabs together advance bit-identically to the single domain. Periodic
 * outer faces of the slab axis make the last and the first rank neighbours.
 * mc_set_slab_decomposition is collective (every rank calls it) and blocks
 * until all have joined. NCCL (libnccl.so.2) is loaded when first needed.
 * No counterpart in the reference, which runs one domain. */
mc_status mc_slab_unique_id(uint8_t* id /* 128 bytes */);
mc_status mc_set_slab_decomposition(mc_ctx* ctx, const uint8_t* id, int32_t rank, int32_t world);
/* 2D slabs (on by default): each stage runs as two launches, the tile rows
 * that read ghost rows or write the layers that are sent, and the other
 * rows on a second internal stream, and the exchange of the first runs
 * beside the second; the next stage's border rows wait for it. Same results
 * either way. Not taken with a non-ideal EOS or a user boundary hook. */
mc_status mc_set_slab_overlap(mc_ctx* ctx, int32_t enable);

/* ---- Non-ideal equations of state --------------------------------------------
 *
 * The EOS kinds of the reference (EosType ordinals, source/Eos.hpp:16-21);
 * the DexRT-coupled kind is out of scope. */
typedef enum {
    MC_EOS_IDEAL = 0,
    MC_EOS_ANALYTIC_LTE_H = 1,   /* source/AnalyticLteH.hpp */
    MC_EOS_TABULATED_LTE_H = 2   /* source/TabulatedLteH.hpp */
} mc_eos_type;

/* Table of the tabulated LTE hydrogen EOS (the NetCDF variables the
 * reference reads, source/TabulatedLteH.hpp:30-58): ionisation fraction y
 * and log10 T on a grid uniform in log10(eint / rho) (fastest) and
 * log10(rho); host arrays of n_rho x n_eint_rho values, copied. */
typedef struct {
    double log_eint_rho_start, log_eint_rho_step;
    int32_t n_eint_rho;
    double log_rho_start, log_rho_step;
    int32_t n_rho;
    const double* y_table;
    const double* log_T_table;
} mc_eos_table;

/* Selects the EOS, as Eos::init does (source/Eos.cpp:11-86; avg_mass is the
 * config key eos.avg_mass, include_ionisation_energy
 * eos.include_ionisation_energy, table the file eos.table_path holds). For a
 * non-ideal kind the update runs ahead of every stage on the stage's input
 * state, cells and ghosts (compute_hydro_fluxes, source/Hydro.cpp:326-328):
 * the analytic kind computes the temperature and ionisation fraction fields
 * by bisection and leaves the state alone; the tabulated kind interpolates
 * them and shifts the energy by the ionisation energy of the change of y
 * since the previous update (the step-start state keeps its energy, as the
 * reference's Q_old copy does). Results agree with the reference to the
 * rounding of pow / exp / log10. */
mc_status mc_set_eos(mc_ctx* ctx, int32_t type, double avg_mass, int32_t include_ionisation_energy,
                     const mc_eos_table* table);
/* One EOS update of Q in place, as setup_sim makes before the first step
 * (source/SetupModules.hpp:253-255). */
mc_status mc_update_eos(mc_ctx* ctx, double* Q, void* stream);
/* Copies the fields of the last update, y_space and T_space (zc*yc*xc
 * doubles each, the layout of one variable of Q), to y and T (device or
 * host memory; either may be NULL). */
mc_status mc_get_eos_fields(mc_ctx* ctx, double* y, double* T, void* stream);

/* Fills W (device memory, the layout of Q) with the primitive state the
 * reference's State.W holds after its last time_step: global_cons_to_prim
 * (source/Hydro.cpp:8-53) of the input of the step's last stage, over every
 * cell, ghosts included, tracers as mass fractions. The library keeps that
 * stage input in its own stage buffer. Before the context's first step, Q
 * (the caller's state) is converted instead. What write_output stores as
 * "W" (source/Output.cpp:226-229). */
mc_status mc_get_prim(mc_ctx* ctx, const double* Q, double* W, void* stream);

/* Registers the gravity source term (setup_gravity,
 * source/SourceTerms/Gravity.cpp:44-70; config keys sources.gravity.x/y/z):
 * every stage adds dt * (0, rho g_x, rho g_y, rho g_z, m . g) to the hydro
 * variables of each interior cell, evaluated from the stage's input state
 * (Gravity.cpp:16-41 with the stage updates of source/TimeStepping.cpp).
 * Components beyond num_dim are ignored. enabled = 0 removes it (the
 * default: no source term, S = 0). */
mc_status mc_set_gravity(mc_ctx* ctx, int32_t enabled, double gx, double gy, double gz);

/* fill_bcs (source/Boundaries.hpp:121-149): fill every ghost cell of Q from
 * the interior for the built-in boundary kinds, x then y then z. */
mc_status mc_fill_bcs(mc_ctx* ctx, double* Q, void* stream);

/* compute_dt (source/Hydro.cpp:209-242): min over every cell, ghosts
 * included, of dx / (c_s + |v|), times max_cfl, then, when clock is not NULL,
 * the output-time clamp. Waits for the stream; writes the result to *dt_out. */
mc_status mc_compute_dt(mc_ctx* ctx, const double* Q, const mc_clock* clock, double* dt_out,
                        void* stream);

/* time_step (source/TimeStepping.cpp:39-308): one SSPRK step of size dt in
 * place on Q (ghosts filled on entry and on exit). Each stage is one fused
 * kernel (two in 3D). The CFL minimum of the new state is reduced in the
 * last stage and can be read with mc_last_cfl_min. */
mc_status mc_time_step(mc_ctx* ctx, double* Q, double dt, void* stream);

/* compute_dt + time_step (source/main.cpp:55-56) on a state that lives in
 * host memory, for a caller that keeps it there between steps (a CPU build
 * of Mosscap handing its step to the GPU): Q_host is copied into Q (a device
 * array of the same layout, the caller's), dt is formed as mc_compute_dt
 * forms it under *clock (no output clamp when clock is NULL), one step is
 * taken, the result is copied back into Q_host and *dt_out = dt. Results are
 * those of the copies plus mc_compute_dt plus mc_time_step. In 2D (ideal
 * EOS, no user or CFL hook, no slab exchange, more than 30 interior rows)
 * the copies overlap the step: stage 0's fluxes are computed band of rows by
 * band as the state arrives and dt is applied once all of it is in; the last
 * stage runs band by band, each band copied back behind it. Q_host should be
 * pinned (cudaHostAlloc) for the copies to overlap. *clock is not advanced.
 * A dt that is not positive and finite fails with MC_ERR_INVALID_ARGUMENT
 * and no step. Waits for the stream. */
mc_status mc_step_host(mc_ctx* ctx, double* Q_host, double* Q, const mc_clock* clock, double* dt_out,
                       void* stream);

/* The main loop of source/main.cpp:54-72 on the device: up to max_steps of
 * { dt = compute_dt; time_step(dt); time += dt } stopping after the step
 * that reaches max_time or an output time (prev_output_time + output_delta),
 * where prev_output_time becomes time. The first dt is computed from Q; later
 * ones are fused into each step's last stage. dt and time never leave the
 * GPU inside the loop; on return (after waiting for the stream) *clock holds
 * the new clock, *steps_done the steps taken and, if dt_log is not NULL,
 * dt_log[0..steps_done) the dt of each step. */
mc_status mc_advance(mc_ctx* ctx, double* Q, mc_clock* clock, int64_t max_steps,
                     int64_t* steps_done, double* dt_log, void* stream);

/* Raw CFL minimum (before max_cfl) of the state written by the last
 * mc_time_step / mc_advance step. Waits for the stream. */
mc_status mc_last_cfl_min(mc_ctx* ctx, double* cfl_min, void* stream);

/* Physics flags (MC_FLAG_*) accumulated since the last call; clears them.
 * Waits for the stream. */
mc_status mc_get_status(mc_ctx* ctx, uint32_t* flags, void* stream);

/* Kernel timing with CUDA events recorded on the launch stream around every
 * stage kernel (kind 0: the fused stage kernel, or in 3D its x-y plane pass;
 * kind 1: the 3D z pass). mc_profile_stages(ctx, 1) starts recording (and
 * clears earlier records), 0 stops. mc_stage_time waits for the recorded
 * events and returns the summed kernel time in milliseconds and the number of
 * launches of that kind. */
mc_status mc_profile_stages(mc_ctx* ctx, int32_t enable);
mc_status mc_stage_time(mc_ctx* ctx, int32_t kind, double* total_ms, int64_t* launches);

/* ---- Batches of independent problems ---------------------------------------
 *
 * Thousands of independent 1D / 2D problems of uneven size advance together:
 * every step of the whole batch is one persistent kernel launch per SSPRK
 * stage (the 2D problems' tiles and the 1D problems' warp tasks in one work
 * list) plus one clock launch, and the step is replayed from a captured CUDA
 * graph. (The autotuner may instead split each stage into a launch over the
 * tiles and one over the 1D tasks, when that measures more than 5 % faster.) Each problem runs the
 * reference's main loop on its own (source/main.cpp:54-72): its own CFL dt,
 * clamped to its own output times and max_time; outputs only advance its
 * clock (prev_output_time = time); a problem that reaches max_time stops.
 * No counterpart as such in the reference (which runs one problem). */
typedef struct mc_batch mc_batch;

typedef struct {
    mc_grid grid;     /* num_dim 1 or 2, num_tracers 0, built-in boundary kinds except constant */
    int64_t offset;   /* offset in doubles of this problem's Q inside the caller's pool */
    double max_cfl;   /* this problem's CFL number */
    mc_clock clock;   /* initial clock */
} mc_batch_problem;

/* The scheme (reconstruction, limiter, solver, stepper, precision, gamma) is
 * shared; scheme->max_cfl is ignored in favour of each problem's. pool_doubles
 * is the size of the caller's pool; the batch allocates two more of that size
 * for its stage buffers. */
mc_status mc_batch_create(const mc_batch_problem* problems, int32_t n, const mc_scheme* scheme,
                          int64_t pool_doubles, mc_batch** out);
mc_status mc_batch_destroy(mc_batch* batch);
/* Fill every problem's ghost cells (fill_bcs per problem). */
mc_status mc_batch_fill_bcs(mc_batch* batch, double* pool, void* stream);
/* Autotuner: times a stage on this pool with CUDA events in both forms (one
 * launch over all work items; a launch over the 2D problems' tiles plus one
 * over the 1D problems' warp tasks) for every candidate schedule (persistent
 * grid size, static or dynamic work distribution, segments per 1D warp task)
 * and keeps the fastest schedule of each form, and the one-launch form
 * unless the split form is more than 5 % faster. Leaves the pool unchanged.
 * Waits for the stream. */
mc_status mc_batch_tune(mc_batch* batch, double* pool, void* stream);
/* Up to `steps` steps of every unfinished problem, each with its own dt, on
 * the device (graph replay). The first call computes every problem's first
 * dt from its state. */
mc_status mc_batch_advance(mc_batch* batch, double* pool, int64_t steps, void* stream);
/* Per-problem clocks, steps taken and MC_FLAG_* status (NULL to skip any).
 * Waits for the stream. */
mc_status mc_batch_clocks(mc_batch* batch, mc_clock* clocks, int64_t* steps, uint32_t* status, void* stream);
/* The schedule in use: grid size in CTAs and 1 if dynamic, of the launch over
 * all work items (one launch per stage) or of the launch over the 2D tiles
 * (two); 1D segments per warp task. */
mc_status mc_batch_schedule(const mc_batch* batch, int32_t* grid, int32_t* dynamic, int32_t* segs_per_task);
/* Launches per stage: 1 (the default: one launch over all work items) or 2
 * (the tiles, then the 1D tasks). The setter overrides the autotuner's
 * choice until the next mc_batch_tune. */
mc_status mc_batch_set_stage_launches(mc_batch* batch, int32_t launches);
mc_status mc_batch_stage_launches(const mc_batch* batch, int32_t* launches);

/* ---- Discrete adjoint --------------------------------------------------------
 *
 * Reverse-mode derivative of n steps of the 2D scheme (WENO5-Z + HLLC +
 * SSPRK3, FP64, periodic faces): the exact vector-Jacobian product of the
 * discrete map the forward kernels compute, including each step's dt (the
 * CFL minimum, through its arg-min cell) and gamma. Reconstruction weights,
 * HLLC wave-speed choices and min / max / |x| are differentiated along the
 * branch the forward computation takes. The forward run stores the state
 * every checkpoint_every steps; the reverse sweep recomputes each segment
 * from its checkpoint. No counterpart in the reference. */
typedef struct mc_adjoint mc_adjoint;

mc_status mc_adjoint_create(const mc_grid* grid, const mc_scheme* scheme, int32_t checkpoint_every,
                            mc_adjoint** out);
mc_status mc_adjoint_destroy(mc_adjoint* adj);
/* Advance Q (ghosts filled) by exactly n_steps steps in place, each with
 * dt = compute_dt under *clock (which must not reach max_time within the run),
 * recording dt, the CFL minimum and the checkpoints. */
mc_status mc_adjoint_forward(mc_adjoint* adj, double* Q, const mc_clock* clock, int64_t n_steps, void* stream);
/* lambda: on entry dJ/dQ of the final state, on exit dJ/dQ of the initial
 * state (interior cells; the layout of Q). *dgamma (if not NULL) receives
 * dJ/dgamma through the steps (the initial state held fixed). Waits for the
 * stream when dgamma is not NULL. */
mc_status mc_adjoint_backward(mc_adjoint* adj, double* lambda, double* dgamma, void* stream);

/* Slab decomposition of the adjoint over ranks (one GPU per rank). The
 * periodic 2D problem is split along y into one slab per rank, ranks in y
 * order (rank 0 the lowest rows, at least 5 rows each); each rank creates
 * its mc_adjoint for its own slab (grid = its rows with ghost layers) and
 * joins before mc_adjoint_forward, with the id of mc_slab_unique_id
 * (collective, as mc_set_slab_decomposition). Then:
 *   forward: the ghost rows between slabs are exchanged after every stage
 *     (and once on entry, so the caller's y ghosts are not read) and every dt
 *     is the all-reduce MIN of the ranks' CFL minima: the slabs together
 *     advance bit-identically to the single domain;
 *   backward: the reverse sweep is the transpose of that exchange. The
 *     cotangent of a cell comes from the faces whose stencils read it,
 *     including the faces just across a slab border, which a neighbour's
 *     cells own: before every stage's product each rank receives the 5
 *     bordering rows of the stage input and the 3 bordering rows of the
 *     stage cotangent from each neighbour and recomputes those faces'
 *     contributions to its own cells itself (a gather rather than a
 *     scatter-and-add of ghost cotangents, so no cell is written by two
 *     ranks). Each step's dt sensitivity is summed over the ranks and routed
 *     to the lowest-index global CFL arg-min cell, on the rank that owns it;
 *     dJ/dgamma is summed over the ranks at the end.
 * Per-cell arithmetic is that of the single domain; the sums of the dt and
 * gamma sensitivities change order with the partition (rounding-level
 * differences with world > 1; bit-identical with world = 1). */
mc_status mc_adjoint_set_slab_decomposition(mc_adjoint* adj, const uint8_t* id, int32_t rank, int32_t world);

/* The same decomposition with the caller moving the data: the library calls
 * fn(user, op, bufs, count, stream) wherever it would call NCCL, with device
 * buffers and work enqueued on `stream` before it; fn returns 0 on success,
 * any other value fails the library call with MC_ERR_CUDA. Every rank makes
 * the same calls in the same order.
 *   MC_COMM_HALO: bufs = {send_lo, send_hi, recv_lo, recv_hi}, count
 *     doubles each: send_lo to the rank below (rank-1, periodic), which
 *     receives it in its recv_hi; send_hi to the rank above, into its recv_lo.
 *   MC_COMM_MIN_U64 / MC_COMM_SUM_F64 / MC_COMM_MIN_I64: bufs[0], count
 *     elements, all-reduced in place. */
typedef enum {
    MC_COMM_HALO = 0,
    MC_COMM_MIN_U64 = 1,
    MC_COMM_SUM_F64 = 2,
    MC_COMM_MIN_I64 = 3
} mc_comm_op;
typedef int32_t (*mc_comm_fn)(void* user, int32_t op, void* const* bufs, int64_t count, void* stream);
mc_status mc_adjoint_set_slab_hook(mc_adjoint* adj, mc_comm_fn fn, void* user, int32_t rank, int32_t world);

/* Tangent-linear (forward-mode) derivative of n_steps steps of the scheme the
 * adjoint covers (2D, WENO5-Z + HLLC, FP64, periodic faces, any stepper),
 * with dt = compute_dt under *clock each step: Q (device, ghosts filled or
 * not) is advanced in place, bit-identical to the forward kernels, and dQ
 * (device, n_dirs states in the layout of Q: on entry the tangents of the
 * initial state, on exit those of the final state) together with dgamma
 * (host, n_dirs values: the tangent of gamma in each direction) is carried
 * along by dual-number evaluation of the forward arithmetic, each branch
 * (WENO weights, HLLC wave speeds, min / max / |x|, the CFL arg-min cell)
 * taken as the forward run takes it. dt's derivative is that of
 * max_cfl * dx / (c_s + |v|) at the lowest-index cell holding the CFL
 * minimum, zero when the output clamp fixes dt. Allocates its own scratch;
 * waits for the stream; *clock returns advanced. An independent check of
 * mc_adjoint_backward: <lambda, J dQ> computed both ways must agree. No
 * counterpart in the reference. */
mc_status mc_tangent_linear(const mc_grid* grid, const mc_scheme* scheme, double* Q, double* dQ,
                            const double* dgamma, int32_t n_dirs, mc_clock* clock, int64_t n_steps, void* stream);

/* One SSPRK step in place on Q, like mc_time_step, without a context and
 * without allocating any device memory. No counterpart in the reference.
 *
 * For callers that cannot call cudaMalloc: a code whose device memory is
 * owned by a pool allocator sized at start-up (Mosscap itself allocates
 * through a YAKL/Kokkos pool), or one that must not call cudaMalloc/cudaFree
 * mid-run because those calls synchronise the device. The stage buffers
 * come from one static device array of 16 MiB that every GPU loading the
 * library holds until the process exits; a problem needs
 * 2 x (2+num_dim+num_tracers) x xc x yc x zc doubles (plus
 * (2+num_dim+num_tracers) x nx x ny x nz in 3D) and is rejected with
 * MC_ERR_OUT_OF_MEMORY when that exceeds 16 MiB (a 4-variable 2D grid with
 * 3 ghosts fits up to 506 x 506 interior cells). All faces must be built-in kinds
 * (no user hook without a context). The first call on a device looks up the
 * array's device address with that device current; make that first call
 * before any stream capture. All calls share the array and its contents
 * persist between calls: calls whose work overlaps on the GPU race and must
 * not be issued. The CFL minimum and status flags of the call go to a block
 * shared by all such calls and are not reported. */
mc_status mc_time_step_noalloc(const mc_grid* grid, const mc_scheme* scheme, double* Q, double dt,
                               void* stream);

/* Number of kernel launches issued by this context since it was created. */
int64_t mc_launch_count(const mc_ctx* ctx);

/* Diagnostic: out[i] = the reciprocal the adjoint's reverse sweep uses for
 * x[i] (device arrays of n doubles), so that its error against IEEE 1/x can
 * be measured. No counterpart in the reference. */
mc_status mc_debug_reverse_reciprocal(const double* x, double* out, int64_t n, void* stream);

/* Message of the last failed call on this thread (static storage). */
const char* mc_last_error(void);

int32_t mc_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MOSSCAP_B200_H */
