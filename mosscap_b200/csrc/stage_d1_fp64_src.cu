// Stage-kernel launchers, 1D, FP64 (compiled with -fmad=false: bit-exact), with the gravity
// source term registered.
#define MC_DIM 1
#define MC_REAL double
#define MC_SRC 1
#define MC_LAUNCH_NAME launch_stage_d1_fp64_src
#include "launch_impl.cuh"
