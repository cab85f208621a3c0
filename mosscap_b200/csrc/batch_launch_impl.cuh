// Launchers of the batched stage kernel for one compute type (MC_REAL);
// batch_stage_fp64.cu and batch_stage_fp32.cu define the macros and include
// this file.
#pragma once

#include <cuda_runtime.h>

#include "batch_kernels.cuh"
#include "batch_launch.h"

#ifndef MC_REAL
#error "MC_REAL must be defined"
#endif

namespace mc {
namespace {

using Real = MC_REAL;

template <int REC, int LIM, int RS, int PART>
cudaError_t launch_batch_part(const BatchStageParams& bp, int grid, cudaStream_t s, int* occupancy) {
    auto k = batch_stage_kernel<REC, LIM, RS, Real, PART>;
    const size_t sm = batch_smem_bytes<REC, Real, PART>();
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) {
        return e;
    }
    if (occupancy) {
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, k, batch_threads<PART>(), sm);
    }
    k<<<grid, batch_threads<PART>(), sm, s>>>(bp);
    return cudaGetLastError();
}

template <int REC, int LIM, int RS>
cudaError_t launch_batch_one(const BatchStageParams& bp, int part, int grid, cudaStream_t s, int* occupancy) {
    switch (part) {
        case kPart2d:
            return launch_batch_part<REC, LIM, RS, kPart2d>(bp, grid, s, occupancy);
        case kPart1d:
            return launch_batch_part<REC, LIM, RS, kPart1d>(bp, grid, s, occupancy);
        default:
            return launch_batch_part<REC, LIM, RS, kPartAll>(bp, grid, s, occupancy);
    }
}

template <int REC, int LIM>
cudaError_t batch_by_solver(const BatchStageParams& bp, int rs, int part, int grid, cudaStream_t s, int* occ) {
    switch (rs) {
        case kRusanov:
            return launch_batch_one<REC, LIM, kRusanov>(bp, part, grid, s, occ);
        case kHll:
            return launch_batch_one<REC, LIM, kHll>(bp, part, grid, s, occ);
        default:
            return launch_batch_one<REC, LIM, kHllc>(bp, part, grid, s, occ);
    }
}

} // namespace

cudaError_t MC_BATCH_LAUNCH_NAME(const BatchStageParams& bp, int rec, int lim, int rs, int part, int grid,
                                 cudaStream_t s, int* occupancy) {
    switch (rec) {
        case kFog:
            return batch_by_solver<kFog, kMonotonizedCentral>(bp, rs, part, grid, s, occupancy);
        case kMuscl:
            switch (lim) {
                case kVanLeer:
                    return batch_by_solver<kMuscl, kVanLeer>(bp, rs, part, grid, s, occupancy);
                case kMonotonizedCentral:
                    return batch_by_solver<kMuscl, kMonotonizedCentral>(bp, rs, part, grid, s, occupancy);
                default:
                    return batch_by_solver<kMuscl, kMinmod>(bp, rs, part, grid, s, occupancy);
            }
        case kPpm:
            switch (lim) {
                case kVanLeer:
                    return batch_by_solver<kPpm, kVanLeer>(bp, rs, part, grid, s, occupancy);
                case kMonotonizedCentral:
                    return batch_by_solver<kPpm, kMonotonizedCentral>(bp, rs, part, grid, s, occupancy);
                default:
                    return batch_by_solver<kPpm, kMinmod>(bp, rs, part, grid, s, occupancy);
            }
        default:
            return batch_by_solver<kWeno5z, kMonotonizedCentral>(bp, rs, part, grid, s, occupancy);
    }
}

} // namespace mc
