// Stage-kernel launchers, 3D, FP64 (compiled with -fmad=false: bit-exact).
#define MC_DIM 3
#define MC_REAL double
#define MC_LAUNCH_NAME launch_stage_d3_fp64
#include "launch_impl.cuh"
