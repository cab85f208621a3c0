// Batched stage-kernel launchers, FP32 compute form.
#define MC_REAL float
#define MC_BATCH_LAUNCH_NAME launch_batch_stage_fp32
#include "batch_launch_impl.cuh"
