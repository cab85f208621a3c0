// Host-side declarations of the batched-stage launchers.
#pragma once

#include <cuda_runtime.h>

#include "batch_kernels.cuh"

namespace mc {

// Launch one part (kPart2d: the 2D tiles, kPart1d: the 1D task bundles,
// kPartAll: both) of one batched stage on `grid` CTAs; with occupancy != NULL, only report the
// resident CTAs per SM of that kernel instead.
cudaError_t launch_batch_stage_fp64(const BatchStageParams& bp, int rec, int lim, int rs, int part, int grid,
                                    cudaStream_t s, int* occupancy);
cudaError_t launch_batch_stage_fp32(const BatchStageParams& bp, int rec, int lim, int rs, int part, int grid,
                                    cudaStream_t s, int* occupancy);

} // namespace mc
