/*
 * Oracle test infrastructure, not product code.
 *
 * One C interface, implemented twice:
 *   - oracle/ref_harness.cpp wraps Mosscap's own hydro hot-path sources
 *     (compiled from the reference tree against oracle/ref_shim) and builds
 *     oracle/_ref/libmosscap_ref.so;
 *   - oracle/mosscap_oracle.c is a plain-C restatement of the same algorithm
 *     and builds oracle/liboracle_port.so.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
 * either library, as the checker.
 *
 * Enum values are the reference's ordinals: Reconstruction / SlopeLimiter
 * (source/Reconstruct.hpp:10-27), RiemannSolver (source/Riemann.hpp:10-14),
 * TimeStepScheme (source/TimeStepping.hpp:10-14), BoundaryType
 * (source/State.hpp:62-70).
 */
#ifndef MOSSCAP_ORACLE_H
#define MOSSCAP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t num_dim;       /* 1, 2 or 3 */
    int32_t nx, ny, nz;    /* interior cells per axis (ny, nz ignored above num_dim) */
    int32_t ng;            /* ghost cells on each side of every active axis */
    int32_t num_tracers;   /* passive scalars after the 2+num_dim hydro vars */
    double dx;             /* cell width (same on every axis) */
    double loc[3];         /* State::loc, lower corner of the first interior cell */
    int32_t bc[6];         /* xs, xe, ys, ye, zs, ze (BoundaryType ordinals) */
    double bc_const[6][5]; /* conserved values for Constant boundaries, Cons<num_dim> order */
    int32_t reconstruction, slope_limiter, riemann_solver, time_stepper;
    double gamma;
    double max_cfl;
    double max_time;
    double output_delta;   /* OutputConfig::delta, drives the dt clamp */
} moracle_config;

void* moracle_create(const moracle_config* cfg);
void moracle_destroy(void* sim);
/* Number of doubles in Q: (2+num_dim+num_tracers) * zc * yc * xc. */
int64_t moracle_state_size(void* sim);
void moracle_set_Q(void* sim, const double* q);
void moracle_get_Q(void* sim, double* q_out);
/* Primitive state left by the last conversion (Hydro.cpp global_cons_to_prim). */
void moracle_get_W(void* sim, double* w_out);
void moracle_fill_bcs(void* sim);
/* Simulation::compute_dt: CFL minimum over every cell times max_cfl, then the
 * clamp to the next output time (Hydro.cpp:209-242). */
double moracle_compute_dt(void* sim);
/* Raw CFL minimum over every cell, before max_cfl and the clamp. */
double moracle_cfl_min(void* sim);
/* Simulation::time_step(sim, dt) (TimeStepping.cpp). */
void moracle_time_step(void* sim, double dt);
/* The main loop of main.cpp:54-72 without I/O: while time < max_time and
 * fewer than max_steps steps were taken: dt = compute_dt; time_step(dt);
 * when time >= prev_output_time + delta set prev_output_time = time.
 * Writes each dt to dt_log (if not NULL); returns the number of steps. */
int64_t moracle_run(void* sim, int64_t max_steps, double* dt_log);
double moracle_get_time(void* sim);
/* Sets the clock: current time and the time of the previous output. */
void moracle_set_clock(void* sim, double time, double prev_output_time);
void moracle_set_num_threads(int n);
/* Registers the gravity source term (setup_gravity,
 * source/SourceTerms/Gravity.cpp:44-70) with acceleration (gx, gy, gz);
 * enabled = 0 leaves the simulation without source terms. */
void moracle_set_gravity(void* sim, int enabled, double gx, double gy, double gz);

/* Table of the tabulated LTE hydrogen EOS (source/TabulatedLteH.hpp:10-27):
 * y and log10 T on a grid uniform in log10(eint / rho) (x, fastest) and
 * log10(rho) (y); arrays [n_rho][n_eint_rho]. */
typedef struct {
    double log_eint_rho_start, log_eint_rho_step;
    int32_t n_eint_rho;
    double log_rho_start, log_rho_step;
    int32_t n_rho;
    const double* y_table;
    const double* log_T_table;
} moracle_eos_table;
/* Selects the EOS (EosType ordinals, source/Eos.hpp:16-21): 0 ideal, 1
 * analytic LTE hydrogen (include_ionisation_energy as the config key), 2
 * tabulated LTE hydrogen (table copied). avg_mass is eos.avg_mass. Sets
 * Simulation::update_eos as Eos::init does (source/Eos.cpp:40-86), which
 * compute_hydro_fluxes runs ahead of every stage. Returns 0, or -1 for an
 * unknown type or a missing table. */
int moracle_set_eos(void* sim, int type, double avg_mass, int include_ionisation_energy,
                    const moracle_eos_table* table);
/* One update_eos call, as setup_sim makes before the first step
 * (source/SetupModules.hpp:253-255). */
void moracle_update_eos(void* sim);
/* The EOS fields y_space and T_space, zc * yc * xc values each. */
void moracle_get_eos_fields(void* sim, double* y, double* T);
/* Number of conditions on which the reference would have aborted. */
long long moracle_abort_count(void);

#ifdef __cplusplus
}
#endif

#endif
