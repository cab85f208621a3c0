// Stage-kernel launchers, 2D, FP32 compute form.
#define MC_DIM 2
#define MC_REAL float
#define MC_LAUNCH_NAME launch_stage_d2_fp32
#include "launch_impl.cuh"
