// Oracle test infrastructure, not product code.
//
// Runs the reference's own Simulation twice from one initial state: once
// with the hooks the reference installs (source/Hydro.cpp:244-323,
// source/TimeStepping.cpp:96-114,193-211,311-328), once after
// mosscap_b200::install() (include/mosscap_b200_hooks.hpp) has replaced them
// with the B200 library, and drives both with the reference's main loop
// (moracle_run, as source/main.cpp:54-72 does). The Simulation is built as
// oracle/ref_harness.cpp builds it, with the shim's memDevice arrays in CUDA
// managed memory, so that sim.state.Q is device memory as in Mosscap's CUDA
// build. Both results go to files that tests/test_hooks_adapter.py compares
// bit for bit.
//
//   adapter_check <dir> <steps> [user_bc]
//
// reads <dir>/config.bin (one moracle_config), <dir>/q0.bin (the initial Q)
// and, if present, <dir>/gravity.bin (three doubles: the gravity source
// term's acceleration); writes ref_{q,w,dt}.bin and lib_{q,w,dt}.bin and
// prints one line of JSON with both clocks. With `user_bc`, both Simulations
// get the same Mosscap-style user_bc: an inflow state on the x-start face
// (which must be of kind UserFn) that also reads sim.dt_sub.
#include "Hydro.hpp"
#include "TimeStepping.hpp"
#include "Boundaries.hpp"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "moracle.h"
#include "mosscap_b200_hooks.hpp"

Mosscap::Simulation* moracle_simulation(void* p);  // oracle/ref_harness.cpp

namespace {

std::vector<char> read_file(const std::string& path, bool required) {
    std::vector<char> out;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) {
        if (required) {
            std::fprintf(stderr, "adapter_check: cannot open %s\n", path.c_str());
            std::exit(2);
        }
        return out;
    }
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    out.resize(size_t(n));
    if (n > 0 && std::fread(out.data(), 1, size_t(n), f) != size_t(n)) {
        std::fprintf(stderr, "adapter_check: short read of %s\n", path.c_str());
        std::exit(2);
    }
    std::fclose(f);
    return out;
}

void write_file(const std::string& path, const void* data, size_t bytes) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(data, 1, bytes, f) != bytes) {
        std::fprintf(stderr, "adapter_check: cannot write %s\n", path.c_str());
        std::exit(2);
    }
    std::fclose(f);
}

// A user boundary of the kind a Mosscap problem generator installs: the
// ghost cells of the x-start face (all of them, edges and corners included)
// take a fixed inflow state whose density follows sim.dt_sub. In Mosscap's
// CUDA build a user_bc fills device memory with a device loop; the shim's
// loops run on the host, so the ghost runs are written with cudaMemcpy, which
// reaches the library's device stage buffers as well as managed memory.
void inflow_user_bc(const Mosscap::Simulation& sim) {
    const auto& Q = sim.state.Q;
    const auto& sz = sim.state.sz;
    const int nd = sim.num_dim;
    const double gamma = sim.eos.gamma;
    const double rho = 1.25 + 1e-3 * double(sim.dt_sub);
    const double vx = 0.35, vy = -0.1, vz = 0.05, p = 0.9;
    double v2 = vx * vx;
    double q[5];
    q[0] = rho;
    q[1] = rho * vx;
    int ie = 2;
    if (nd > 1) {
        q[2] = rho * vy;
        v2 += vy * vy;
        ie = 3;
    }
    if (nd > 2) {
        q[3] = rho * vz;
        v2 += vz * vz;
        ie = 4;
    }
    q[ie] = p / (gamma - 1.0) + 0.5 * rho * v2;
    std::vector<double> run(static_cast<size_t>(sz.ng));
    for (int v = 0; v <= ie; ++v) {
        std::fill(run.begin(), run.end(), q[v]);
        for (int k = 0; k < sz.zc; ++k) {
            for (int j = 0; j < sz.yc; ++j) {
                if (cudaMemcpy(&Q(v, k, j, 0), run.data(), sizeof(double) * run.size(), cudaMemcpyDefault) !=
                    cudaSuccess) {
                    std::fprintf(stderr, "adapter_check: user_bc copy failed\n");
                    std::exit(3);
                }
            }
        }
    }
}

} // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: adapter_check <dir> <steps> [user_bc]\n");
        return 2;
    }
    const std::string dir = argv[1];
    const long steps = std::atol(argv[2]);
    const bool with_user_bc = argc > 3 && std::string(argv[3]) == "user_bc";
    const std::vector<char> cfg_bytes = read_file(dir + "/config.bin", true);
    if (cfg_bytes.size() != sizeof(moracle_config)) {
        std::fprintf(stderr, "adapter_check: config.bin holds %zu bytes, expected %zu\n", cfg_bytes.size(),
                     sizeof(moracle_config));
        return 2;
    }
    moracle_config cfg;
    std::memcpy(&cfg, cfg_bytes.data(), sizeof(cfg));
    const std::vector<char> q0 = read_file(dir + "/q0.bin", true);
    const std::vector<char> grav = read_file(dir + "/gravity.bin", false);

    void* sims[2] = {moracle_create(&cfg), moracle_create(&cfg)};
    if (!sims[0] || !sims[1]) {
        std::fprintf(stderr, "adapter_check: configuration rejected\n");
        return 2;
    }
    const int64_t n = moracle_state_size(sims[0]);
    if (q0.size() != size_t(n) * sizeof(double)) {
        std::fprintf(stderr, "adapter_check: q0.bin holds %zu bytes, expected %lld\n", q0.size(),
                     (long long)(n * 8));
        return 2;
    }
    double g[3] = {0.0, 0.0, 0.0};
    if (grav.size() == sizeof(g)) {
        std::memcpy(g, grav.data(), sizeof(g));
    }
    for (void* s : sims) {
        if (grav.size() == sizeof(g)) {
            moracle_set_gravity(s, 1, g[0], g[1], g[2]);
        }
        if (with_user_bc) {
            moracle_simulation(s)->user_bc = inflow_user_bc;
        }
        moracle_set_Q(s, reinterpret_cast<const double*>(q0.data()));
        moracle_fill_bcs(s);  // setup's fill_bcs, Mosscap's own (source/main.cpp:52)
    }

    Mosscap::Simulation& lib_sim = *moracle_simulation(sims[1]);
    auto binding = mosscap_b200::install(lib_sim, grav.size() == sizeof(g) ? g : nullptr);

    const char* names[2] = {"ref", "lib"};
    std::vector<double> q(static_cast<size_t>(n)), w(static_cast<size_t>(n));
    std::string json = "{";
    for (int r = 0; r < 2; ++r) {
        std::vector<double> dts(size_t(steps > 0 ? steps : 1));
        const int64_t done = moracle_run(sims[r], steps, dts.data());
        if (cudaDeviceSynchronize() != cudaSuccess) {
            std::fprintf(stderr, "adapter_check: device error after the %s run\n", names[r]);
            return 3;
        }
        moracle_get_Q(sims[r], q.data());
        moracle_get_W(sims[r], w.data());
        const std::string base = dir + "/" + names[r];
        write_file(base + "_q.bin", q.data(), q.size() * sizeof(double));
        write_file(base + "_w.bin", w.data(), w.size() * sizeof(double));
        write_file(base + "_dt.bin", dts.data(), size_t(done) * sizeof(double));
        const Mosscap::Simulation& s = *moracle_simulation(sims[r]);
        char buf[512];
        std::snprintf(buf, sizeof(buf),
                      "%s\"%s\": {\"steps\": %lld, \"current_step\": %lld, \"time\": %.17g, \"dt\": %.17g, "
                      "\"dt_sub\": %.17g, \"prev_output_time\": %.17g}",
                      r ? ", " : "", names[r], (long long)done, (long long)s.current_step, s.time, double(s.dt),
                      double(s.dt_sub), s.out_cfg.prev_output_time);
        json += buf;
    }
    json += "}";
    std::printf("%s\n", json.c_str());
    binding.reset();
    moracle_destroy(sims[0]);
    moracle_destroy(sims[1]);
    return 0;
}
