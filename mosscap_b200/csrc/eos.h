// Launch description of the non-ideal EOS update (eos.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace mc {

constexpr int kEosIdeal = 0;      // EosType::Ideal (source/Eos.hpp:16-21)
constexpr int kEosAnalytic = 1;   // EosType::AnalyticLteH
constexpr int kEosTabulated = 2;  // EosType::TabulatedLteH
constexpr unsigned kFlagEos = 0x10u;  // MC_FLAG_EOS

struct EosLaunch {
    int type;
    const double* q_in;   // the stage input, every cell including ghosts
    double* q_out;        // tabulated: where the shifted state goes (q_in: in place)
    double* y;            // y_space, zc * yc * xc
    double* T;            // T_space
    long long plane;      // zc * yc * xc
    int nvar;
    double gamma, avg_mass;
    int ionisation_e;     // analytic: include the ionisation energy
    // tabulated: the grid and the tables [ny_tab][nx_tab]
    double x_start, x_step, y_start, y_step;
    int nx_tab, ny_tab;
    const double* y_table;
    const double* log_T_table;
    DeviceBlock* blk;     // status flags; with skip_when_done, the device loop's done flag
    int skip_when_done;
};

cudaError_t launch_eos_update(const EosLaunch& L, int ndim, cudaStream_t s);

} // namespace mc
