// Stage-kernel launchers, 3D, FP32 compute form.
#define MC_DIM 3
#define MC_REAL float
#define MC_LAUNCH_NAME launch_stage_d3_fp32
#include "launch_impl.cuh"
