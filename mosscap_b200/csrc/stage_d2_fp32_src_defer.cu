// Stage-kernel launchers, 2D, FP32 (FP32 compute form), with the gravity source term registered:
// the deferred form, whose tiles write only their x+y divergence (mc_step_host).
#define MC_DIM 2
#define MC_REAL float
#define MC_SRC 1
#define MC_DEFER 1
#define MC_LAUNCH_NAME launch_stage_d2_fp32_src_defer
#include "launch_impl.cuh"
