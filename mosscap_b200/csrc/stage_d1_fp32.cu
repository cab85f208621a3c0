// Stage-kernel launchers, 1D, FP32 compute form.
#define MC_DIM 1
#define MC_REAL float
#define MC_LAUNCH_NAME launch_stage_d1_fp32
#include "launch_impl.cuh"
