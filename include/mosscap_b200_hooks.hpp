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
// Mosscap in double precision (fp_t = f64), the ideal EOS, no source term
// other than gravity (whose vector install() must be given, since the
// registered std::function does not expose it); fill_bcs at setup can stay
// Mosscap's own or use mc_fill_bcs.
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

// Replace Simulation::time_step and Simulation::compute_dt. gravity: the
// sources.gravity.{x,y,z} values of the configuration, required when the
// Simulation registered the gravity source term (setup_gravity,
// source/SourceTerms/Gravity.cpp:44-70).
template <class Sim>
Context install(Sim& sim, const double* gravity = nullptr) {
    Context ctx = make_context(sim);
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
    sim.time_step = [ctx](Sim& s, auto dt) {
        check(mc_time_step(ctx.get(), s.state.Q.data(), double(dt), nullptr), "mc_time_step");
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
