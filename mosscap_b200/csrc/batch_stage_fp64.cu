// Batched stage-kernel launchers, FP64 (compiled with -fmad=false: bit-exact).
#define MC_REAL double
#define MC_BATCH_LAUNCH_NAME launch_batch_stage_fp64
#include "batch_launch_impl.cuh"
