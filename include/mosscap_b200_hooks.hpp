// Mosscap-side adapter: installs the B200 library as the hydro hooks of a
// Mosscap Simulation (source/Simulation.hpp:38-62). Header-only; include it
// in a Mosscap translation unit after Simulation.hpp and call
// mosscap_b200::install(sim) after setup_sim (source/SetupModules.hpp:232-262)
// has created the state. The main loop (source/main.cpp:54-72) is unchanged:
//
//   sim.compute_dt(sim)      -> mc_compute_dt (CFL minimum + output clamp)
//   sim.time_step(sim, dt)   -> mc_time_step, then time += dt, step += 1
//                               (source/TimeStepping.cpp:90-92)
//
// The state stays in Mosscap's own device array (sim.state.Q.data()); the
// library owns only its two stage buffers. Requirements: a CUDA build of
// Mosscap in double precision (fp_t = f64), the ideal, analytic or tabulated
// EOS, no source term other than gravity (the gravity vector and a non-ideal
// EOS's settings must be given to install(), since the registered
// std::functions do not expose them); fill_bcs at setup can stay Mosscap's
// own or use mc_fill_bcs.
#pragma once

#include <memory>
#include <stdexcept>
#include <string>

#include "mosscap_b200.h"

namespace mosscap_b200 {

struct ContextDeleter {
    void operator()(mc_ctx* c) const { mc_destroy(c); }
};
using Context = std::shared_ptr<mc_ctx>;

inline void check(mc_status s, const char* where) {
    if (s != MC_OK) {
        throw std::runtime_error(std::string(where) + ": " + mc_last_error());
    }
}

// Build the grid / scheme descriptors from a Mosscap Simulation. Templated on
// the Simulation type so this header does not need Mosscap's headers itself.
template <class Sim>
Context make_context(const Sim& sim) {
    const auto& st = sim.state;
    mc_grid g{};
    g.num_dim = sim.num_dim;
    g.xc = st.sz.xc;
    g.yc = st.sz.yc;
    g.zc = st.sz.zc;
    g.ng = st.sz.ng;
    g.num_tracers = st.num_tracers;
    g.dx = st.dx;
    g.loc[0] = st.loc.x;
    g.loc[1] = st.loc.y;
    g.loc[2] = st.loc.z;
    const auto& b = st.boundaries;
    const int kinds[6] = {int(b.xs), int(b.xe), int(b.ys), int(b.ye), int(b.zs), int(b.ze)};
    const decltype(b.xs_const)* consts[6] = {&b.xs_const, &b.xe_const, &b.ys_const,
                                             &b.ye_const, &b.zs_const, &b.ze_const};
    for (int f = 0; f < 6; ++f) {
        g.bc[f] = kinds[f];
        for (int v = 0; v < 5; ++v) {
            g.bc_const[f][v] = (*consts[f])(v);
        }
    }
    mc_scheme s{};
    s.reconstruction = int(sim.scheme.reconstruction);
    s.slope_limiter = int(sim.scheme.slope_limit);
    s.riemann_solver = int(sim.scheme.riemann_solver);
    s.time_stepper = int(sim.scheme.time_stepper);
    s.precision = MC_PRECISION_FP64;
    s.gamma = sim.eos.gamma;
    s.max_cfl = sim.max_cfl;
    mc_ctx* c = nullptr;
    check(mc_create(&g, &s, &c), "mc_create");
    return Context(c, ContextDeleter{});
}

// The equation of state a Simulation was set up with (Eos::init,
// source/Eos.cpp:11-86): the eos.type ordinal, eos.avg_mass,
// eos.include_ionisation_energy and, for the tabulated kind, the table read
// from eos.table_path. The registered update_eos does not expose them.
struct EosConfig {
    int type;
    double avg_mass;
    bool include_ionisation_energy;
    const mc_eos_table* table;
};

// Replace Simulation::time_step and Simulation::compute_dt. gravity: the
// sources.gravity.{x,y,z} values of the configuration, required when the
// Simulation registered the gravity source term (setup_gravity,
// source/SourceTerms/Gravity.cpp:44-70). eos: required when the Simulation
// has an update_eos (a non-ideal EOS); the library then runs the update
// ahead of every stage and copies y_space / T_space into sim.eos after each
// step, where Mosscap's output and coupling read them.
template <class Sim>
Context install(Sim& sim, const double* gravity = nullptr, const EosConfig* eos = nullptr) {
    Context ctx = make_context(sim);
    const bool non_ideal = bool(sim.update_eos);
    if (non_ideal) {
        if (!eos) {
            throw std::runtime_error("mosscap_b200: a non-ideal EOS needs its EosConfig in install()");
        }
        check(mc_set_eos(ctx.get(), eos->type, eos->avg_mass, eos->include_ionisation_energy ? 1 : 0, eos->table),
              "mc_set_eos");
    }
    bool has_gravity = false;
    for (const auto& term : sim.compute_source_terms) {
        if (term.name != "gravity") {
            throw std::runtime_error("mosscap_b200: unsupported source term \"" + term.name + "\"");
        }
        has_gravity = true;
    }
    if (has_gravity) {
        if (!gravity) {
            throw std::runtime_error("mosscap_b200: the gravity source term needs its vector in install()");
        }
        check(mc_set_gravity(ctx.get(), 1, gravity[0], gravity[1], gravity[2]), "mc_set_gravity");
    }
    sim.time_step = [ctx, non_ideal](Sim& s, auto dt) {
        check(mc_time_step(ctx.get(), s.state.Q.data(), double(dt), nullptr), "mc_time_step");
        if (non_ideal) {
            check(mc_get_eos_fields(ctx.get(), s.eos.y_space.data(), s.eos.T_space.data(), nullptr),
                  "mc_get_eos_fields");
        }
        s.dt = dt;
        s.time += dt;
        s.current_step += 1;
    };
    sim.compute_dt = [ctx](const Sim& s) {
        mc_clock k{s.time, s.max_time, s.out_cfg.prev_output_time, s.out_cfg.delta};
        double dt = 0.0;
        check(mc_compute_dt(ctx.get(), s.state.Q.data(), &k, &dt, nullptr), "mc_compute_dt");
        return dt;
    };
    return ctx;
}

} // namespace mosscap_b200
