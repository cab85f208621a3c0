// Oracle test infrastructure, not product code.
//
// extern "C" harness around Mosscap's own hydro hot path. The reference files
// (source/Hydro.cpp, source/TimeStepping.cpp and the headers they include) are
// compiled unmodified from the reference tree; this file only builds the
// Simulation aggregate the way source/SetupModules.hpp does for the hydro
// part (setup_grid :9-64, setup_boundaries :66-136, setup_hydro_fns
// :138-156, setup_timestepper :158-168, Eos::init_ideal Eos.hpp:37-42,
// setup_output :179-195) and drives it like source/main.cpp:54-72.
// Output is replaced by a function that only records the output time, as
// source/Output.cpp:272 does.
#include "Hydro.hpp"
#include "TimeStepping.hpp"
#include "Boundaries.hpp"
#include "SourceTerms.hpp"
#include "SourceTerms/Gravity.hpp"
#include "AnalyticLteH.hpp"
#include "TabulatedLteH.hpp"
#include "yaml-cpp/yaml.h"

#include <limits>
#include <new>
#include <stdexcept>

#include "moracle.h"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct RefSim {
    Mosscap::Simulation sim{};
};

Mosscap::Simulation& S(void* p) {
    return static_cast<RefSim*>(p)->sim;
}

} // namespace

// The Simulation a handle holds (C++ linkage; oracle/adapter_check.cpp
// installs the C++ hook adapter on it).
Mosscap::Simulation* moracle_simulation(void* p) {
    return &S(p);
}

extern "C" {

void* moracle_create(const moracle_config* c) {
    using namespace Mosscap;
    if (c->num_dim < 1 || c->num_dim > 3) {
        return nullptr;
    }
    if (c->ng < min_ghost_cells(Reconstruction(c->reconstruction))) {
        return nullptr;
    }
    RefSim* r = new (std::nothrow) RefSim();
    if (!r) {
        return nullptr;
    }
    Simulation& sim = r->sim;
    sim.num_dim = c->num_dim;
    sim.current_step = 0;
    sim.time = 0.0;

    // setup_grid (SetupModules.hpp:9-64)
    auto& sz = sim.state.sz;
    sz.ng = c->ng;
    sz.xc = c->nx + 2 * sz.ng;
    sz.yc = 1;
    sz.zc = 1;
    if (sim.num_dim > 1) {
        sz.yc = c->ny + 2 * sz.ng;
    }
    if (sim.num_dim > 2) {
        sz.zc = c->nz + 2 * sz.ng;
    }
    auto& state = sim.state;
    state.dx = c->dx;
    state.loc.x = c->loc[0];
    state.loc.y = c->loc[1];
    state.loc.z = c->loc[2];
    const int n_hydro = get_num_hydro_vars(sim.num_dim);
    state.num_tracers = c->num_tracers;
    const int n_total = n_hydro + c->num_tracers;
    state.Q = Fp4d("Q", n_total, sz.zc, sz.yc, sz.xc);
    state.W = Fp4d("W", n_total, sz.zc, sz.yc, sz.xc);
    sim.recon_scratch.RR = Fp4d("RR", n_total, sz.zc, sz.yc, sz.xc);
    sim.recon_scratch.RL = Fp4d("RL", n_total, sz.zc, sz.yc, sz.xc);
    sim.fluxes.Fx = Fp4d("Fx", n_total, sz.zc, sz.yc, sz.xc);
    if (sim.num_dim > 1) {
        sim.fluxes.Fy = Fp4d("Fy", n_total, sz.zc, sz.yc, sz.xc);
    }
    if (sim.num_dim > 2) {
        sim.fluxes.Fz = Fp4d("Fz", n_total, sz.zc, sz.yc, sz.xc);
    }
    sim.sources.S = Fp4d("S", n_hydro, sz.zc, sz.yc, sz.xc);

    // setup_boundaries (SetupModules.hpp:66-136); unused axes keep Wall as
    // the YAML default would, and are never filled.
    auto& b = state.boundaries;
    BoundaryType* kinds[6] = {&b.xs, &b.xe, &b.ys, &b.ye, &b.zs, &b.ze};
    decltype(b.xs_const)* consts[6] = {&b.xs_const, &b.xe_const, &b.ys_const,
                                       &b.ye_const, &b.zs_const, &b.ze_const};
    for (int f = 0; f < 6; ++f) {
        *kinds[f] = BoundaryType(c->bc[f]);
        for (int v = 0; v < N_HYDRO_VARS<3>; ++v) {
            (*consts[f])(v) = c->bc_const[f][v];
        }
    }

    // setup_hydro_fns / setup_timestepper / setup_eos / setup_output
    sim.scheme.reconstruction = Reconstruction(c->reconstruction);
    sim.scheme.slope_limit = SlopeLimiter(c->slope_limiter);
    sim.scheme.riemann_solver = RiemannSolver(c->riemann_solver);
    sim.scheme.time_stepper = TimeStepScheme(c->time_stepper);
    select_hydro_fns(sim);
    select_timestepper(sim);
    sim.max_cfl = c->max_cfl;
    sim.max_time = c->max_time;
    sim.eos.init_ideal(c->gamma, 1.0, sim);
    sim.out_cfg.delta = c->output_delta;
    sim.out_cfg.output_count = 0;
    // setup_sim writes the initial conditions once at time 0
    // (SetupModules.hpp:258-259), which sets prev_output_time = 0.
    sim.out_cfg.prev_output_time = 0.0;
    sim.write_output = [](Simulation& s) {
        s.out_cfg.prev_output_time = s.time;
        s.out_cfg.output_count += 1;
        return true;
    };
    return r;
}

void moracle_destroy(void* p) {
    delete static_cast<RefSim*>(p);
}

int64_t moracle_state_size(void* p) {
    return S(p).state.Q.size();
}

void moracle_set_Q(void* p, const double* q) {
    auto& Q = S(p).state.Q;
    std::memcpy(Q.data(), q, sizeof(double) * Q.size());
}

void moracle_get_Q(void* p, double* q) {
    auto& Q = S(p).state.Q;
    std::memcpy(q, Q.data(), sizeof(double) * Q.size());
}

void moracle_get_W(void* p, double* w) {
    auto& W = S(p).state.W;
    std::memcpy(w, W.data(), sizeof(double) * W.size());
}

void moracle_fill_bcs(void* p) {
    Mosscap::fill_bcs(S(p));
}

double moracle_compute_dt(void* p) {
    return Mosscap::compute_dt(S(p));
}

double moracle_cfl_min(void* p) {
    auto& sim = S(p);
    const double cfl = sim.max_cfl;
    const double tmax = sim.max_time;
    sim.max_cfl = 1.0;
    sim.max_time = std::numeric_limits<double>::infinity();
    const double m = Mosscap::compute_dt(sim);
    sim.max_cfl = cfl;
    sim.max_time = tmax;
    return m;
}

void moracle_time_step(void* p, double dt) {
    auto& sim = S(p);
    sim.time_step(sim, dt);
}

int64_t moracle_run(void* p, int64_t max_steps, double* dt_log) {
    auto& sim = S(p);
    int64_t n = 0;
    while (sim.time < sim.max_time && n < max_steps) {
        const double dt = Mosscap::compute_dt(sim);
        sim.time_step(sim, dt);
        if (dt_log) {
            dt_log[n] = dt;
        }
        ++n;
        if (sim.time >= sim.out_cfg.prev_output_time + sim.out_cfg.delta) {
            sim.write_output(sim);
        }
    }
    return n;
}

double moracle_get_time(void* p) {
    return S(p).time;
}

void moracle_set_clock(void* p, double time, double prev_output_time) {
    S(p).time = time;
    S(p).out_cfg.prev_output_time = prev_output_time;
}

void moracle_set_gravity(void* p, int enabled, double gx, double gy, double gz) {
    // the reference's own registration, with the configuration
    // sources.gravity.{x,y,z} built in code
    auto& sim = S(p);
    sim.compute_source_terms.clear();
    if (!enabled) {
        return;
    }
    YAML::Node cfg;
    YAML::Node g = cfg.child("sources").child("gravity");
    g.child("x").set(gx);
    g.child("y").set(gy);
    g.child("z").set(gz);
    Mosscap::setup_gravity(sim, cfg);
}

int moracle_set_eos(void* p, int type, double avg_mass, int include_ionisation_energy,
                    const moracle_eos_table* t) {
    using namespace Mosscap;
    Simulation& sim = S(p);
    Eos& eos = sim.eos;
    const auto& sz = sim.state.sz;
    eos.avg_mass = avg_mass;
    if (type == int(EosType::Ideal)) {
        eos.is_constant = true;
        sim.update_eos = nullptr;
        return 0;
    }
    // Eos::init_analytic_lte_h / init_tabulated_lte_h (source/Eos.cpp:40-86),
    // with the table set in code instead of read from NetCDF
    eos.is_constant = false;
    eos.y_space = Fp3d("y_space", sz.zc, sz.yc, sz.xc);
    eos.T_space = Fp3d("T_space", sz.zc, sz.yc, sz.xc);
    eos.y_space = 0.0;
    eos.T_space = 0.0;
    if (type == int(EosType::AnalyticLteH)) {
        AnalyticLteH lte;
        lte.init(include_ionisation_energy != 0);
        sim.update_eos = [lte](const Simulation& s) {
            if (s.num_dim == 1) {
                lte.update_eos<1>(s);
            } else if (s.num_dim == 2) {
                lte.update_eos<2>(s);
            } else {
                lte.update_eos<3>(s);
            }
        };
        return 0;
    }
    if (type == int(EosType::TabulatedLteH) && t && t->y_table && t->log_T_table) {
        TabulatedLteH lte;
        lte.eint_rho_grid = TabulatedLteH::LogSpace{t->log_eint_rho_start, t->log_eint_rho_step, t->n_eint_rho};
        lte.rho_grid = TabulatedLteH::LogSpace{t->log_rho_start, t->log_rho_step, t->n_rho};
        lte.y_table = Fp2d("y_table", t->n_rho, t->n_eint_rho);
        lte.log_T_table = Fp2d("log_T_table", t->n_rho, t->n_eint_rho);
        const size_t n = size_t(t->n_rho) * size_t(t->n_eint_rho);
        std::memcpy(lte.y_table.data(), t->y_table, sizeof(double) * n);
        std::memcpy(lte.log_T_table.data(), t->log_T_table, sizeof(double) * n);
        eos.y_space = -1.0;
        sim.update_eos = [lte](const Simulation& s) {
            if (s.num_dim == 1) {
                lte.update_eos<1>(s);
            } else if (s.num_dim == 2) {
                lte.update_eos<2>(s);
            } else {
                lte.update_eos<3>(s);
            }
        };
        return 0;
    }
    return -1;
}

void moracle_update_eos(void* p) {
    auto& sim = S(p);
    if (sim.update_eos) {
        sim.update_eos(sim);
    }
}

void moracle_get_eos_fields(void* p, double* y, double* T) {
    auto& eos = S(p).eos;
    const size_t n = eos.y_space.size();
    std::memcpy(y, eos.y_space.data(), sizeof(double) * n);
    std::memcpy(T, eos.T_space.data(), sizeof(double) * n);
}

long long moracle_abort_count(void) {
    return Kokkos::abort_count().load();
}

void moracle_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) {
        omp_set_num_threads(n);
    }
#else
    (void)n;
#endif
}

} // extern "C"
