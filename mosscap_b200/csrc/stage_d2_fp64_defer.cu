// Stage-kernel launchers, 2D, FP64 (compiled with -fmad=false: bit-exact):
// the deferred form, whose tiles write only their x+y divergence (mc_step_host).
#define MC_DIM 2
#define MC_REAL double
#define MC_DEFER 1
#define MC_LAUNCH_NAME launch_stage_d2_fp64_defer
#include "launch_impl.cuh"
