// Stage-kernel launchers, 3D, FP32 (FP32 compute form), with the gravity
// source term registered.
#define MC_DIM 3
#define MC_REAL float
#define MC_SRC 1
#define MC_LAUNCH_NAME launch_stage_d3_fp32_src
#include "launch_impl.cuh"
