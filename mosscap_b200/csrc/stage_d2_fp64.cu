// Stage-kernel launchers, 2D, FP64 (compiled with -fmad=false: bit-exact).
#define MC_DIM 2
#define MC_REAL double
#define MC_LAUNCH_NAME launch_stage_d2_fp64
#include "launch_impl.cuh"
