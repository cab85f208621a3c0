// Mosscap-side adapter: installs the B200 library as the hydro hooks of a
// Mosscap Simulation (source/Simulation.hpp:38-62). Header-only; include it
// in a Mosscap translation unit after Simulation.hpp and call
// mosscap_b200::install(sim) after setup_sim (source/SetupModules.hpp:232-262)
// has created the state. The main loop (source/main.cpp:54-72) is unchanged:
//
//   sim.compute_dt(sim)      -> mc_compute_dt (CFL minimum + output clamp)
//   sim.time_step(sim, dt)   -> sim.dt = dt; mc_time_step; W refreshed;
//                               time += dt, step += 1
//                               (source/TimeStepping.cpp:47-48, :90-92)
//   sim.user_bc (if set)     -> called after every stage's ghost fill, as
//                               fill_bcs does (source/Boundaries.hpp:146-148),
//                               with sim.state.Q viewing the stage's buffer
//
// The state stays in Mosscap's own device array (sim.state.Q.data()); the
// library owns only its two stage buffers. Requirements: a CUDA build of
// Mosscap in double precision (fp_t = f64), the ideal, analytic or tabulated
// EOS, no source term other than gravity (the gravity vector and a non-ideal
// EOS's settings must be given to install(), since the registered
// std::functions do not expose them); fill_bcs at setup can stay Mosscap's
// own or use mc_fill_bcs.
//
// user_bc contract. Mosscap calls user_bc at the end of every fill_bcs,
// after the built-in faces. The library writes each stage's output to one of
// its own buffers, so the adapter points sim.state.Q at that buffer (a view,
// restored afterwards), sets sim.dt_sub to the value the reference's stepper
// holds at that fill, and waits for the device before and after the call. A
// user_bc must fill every ghost cell of its MC_BC_USERFN faces, the corner
// and edge ghosts included: the library does not copy stale values into
// those corners the way the reference's per-axis fill does.
#pragma once

#include <cuda_runtime.h>

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

// Options of install().
struct InstallOptions {
    // Refresh sim.state.W after every step with the primitives the
    // reference's W holds at that point (the last stage's input through
    // global_cons_to_prim, source/Hydro.cpp:8-53), which write_output stores
    // (source/Output.cpp:226-229). One conversion pass per step.
    bool refresh_W = true;
};

// What install() leaves behind: the library context and the state the
// forwarded user_bc needs. Keep it alive as long as the hooks are used.
template <class Sim>
struct Installed {
    Context ctx;
    Sim* sim = nullptr;
    int stepper = 0;
    int stage = 0;      // stage fills seen in the step in flight
    double dt = 0.0;
    bool refresh_W = true;
    std::string error;  // set by the forwarded user_bc, raised after the step
};
template <class Sim>
using Binding = std::shared_ptr<Installed<Sim>>;

// sim.dt_sub as the reference's stepper holds it when fill_bcs (and so
// user_bc) runs after stage `stage`: each stepper sets it before a stage
// (source/TimeStepping.cpp: rk2 :49, :70; ssprk3 :126, :147, :167;
// ssprk4 :224, :244, :264, :284) and the fill after a stage comes after the
// next stage's value is set, the last fill after the last one's.
inline double dt_sub_at_fill(int stepper, int stage, double dt) {
    if (stepper == MC_STEPPER_RK2) {
        return 0.5 * dt;
    }
    if (stepper == MC_STEPPER_SSPRK3) {
        return stage == 0 ? 0.25 * dt : (2.0 / 3.0) * dt;
    }
    const int next = stage + 1 < 4 ? stage + 1 : 3;
    return next == 2 ? (1.0 / 6.0) * dt : 0.5 * dt;
}

template <class Sim>
void forward_user_bc(void* user, double* q, void* stream) {
    auto* b = static_cast<Installed<Sim>*>(user);
    Sim& s = *b->sim;
    if (!b->error.empty()) {
        return;
    }
    // the stage kernels run on `stream`; Mosscap's own kernels may not
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) != cudaSuccess) {
        b->error = "stream synchronisation before user_bc failed";
        return;
    }
    auto saved = s.state.Q;
    s.state.Q = decltype(saved)("Q", q, saved.extent(0), saved.extent(1), saved.extent(2), saved.extent(3));
    const auto saved_dt_sub = s.dt_sub;
    s.dt_sub = dt_sub_at_fill(b->stepper, b->stage, b->dt);
    b->stage += 1;
    s.user_bc(s);
    s.state.Q = saved;
    s.dt_sub = saved_dt_sub;
    if (cudaDeviceSynchronize() != cudaSuccess) {
        b->error = "device synchronisation after user_bc failed";
    }
}

// Replace Simulation::time_step and Simulation::compute_dt. gravity: the
// sources.gravity.{x,y,z} values of the configuration, required when the
// Simulation registered the gravity source term (setup_gravity,
// source/SourceTerms/Gravity.cpp:44-70). eos: required when the Simulation
// has an update_eos (a non-ideal EOS); the library then runs the update
// ahead of every stage and copies y_space / T_space into sim.eos after each
// step, where Mosscap's output and coupling read them. A user_bc set on the
// Simulation is forwarded (see the contract above). The Simulation must stay
// at its address while the hooks are in use.
template <class Sim>
Binding<Sim> install(Sim& sim, const double* gravity = nullptr, const EosConfig* eos = nullptr,
                     InstallOptions opt = InstallOptions()) {
    auto b = std::make_shared<Installed<Sim>>();
    b->ctx = make_context(sim);
    b->sim = &sim;
    b->stepper = int(sim.scheme.time_stepper);
    b->refresh_W = opt.refresh_W;
    mc_ctx* ctx = b->ctx.get();
    const bool non_ideal = bool(sim.update_eos);
    if (non_ideal) {
        if (!eos) {
            throw std::runtime_error("mosscap_b200: a non-ideal EOS needs its EosConfig in install()");
        }
        check(mc_set_eos(ctx, eos->type, eos->avg_mass, eos->include_ionisation_energy ? 1 : 0, eos->table),
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
        check(mc_set_gravity(ctx, 1, gravity[0], gravity[1], gravity[2]), "mc_set_gravity");
    }
    if (sim.user_bc) {
        check(mc_set_user_bc(ctx, &forward_user_bc<Sim>, b.get()), "mc_set_user_bc");
    }
    sim.time_step = [b, non_ideal](Sim& s, auto dt) {
        s.dt = dt;
        b->dt = double(dt);
        b->stage = 0;
        check(mc_time_step(b->ctx.get(), s.state.Q.data(), double(dt), nullptr), "mc_time_step");
        if (!b->error.empty()) {
            throw std::runtime_error("mosscap_b200: " + b->error);
        }
        if (b->refresh_W) {
            check(mc_get_prim(b->ctx.get(), s.state.Q.data(), s.state.W.data(), nullptr), "mc_get_prim");
        }
        if (non_ideal) {
            check(mc_get_eos_fields(b->ctx.get(), s.eos.y_space.data(), s.eos.T_space.data(), nullptr),
                  "mc_get_eos_fields");
        }
        s.dt_sub = dt_sub_at_fill(b->stepper, 3, double(dt));
        s.time += dt;
        s.current_step += 1;
    };
    sim.compute_dt = [b](const Sim& s) {
        mc_clock k{s.time, s.max_time, s.out_cfg.prev_output_time, s.out_cfg.delta};
        double dt = 0.0;
        check(mc_compute_dt(b->ctx.get(), s.state.Q.data(), &k, &dt, nullptr), "mc_compute_dt");
        return dt;
    };
    return b;
}

} // namespace mosscap_b200
