// Host-side declarations of the kernel launchers (csrc/*.cu).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace mc {

// The stage plan of each SSPRK driver (source/TimeStepping.cpp: rk2 :39-93,
// ssprk3 :116-190, ssprk4 :213-308): input and output buffer of each stage
// (0 = the caller's Q, 1 = stage buffer A, 2 = stage buffer B) and the stage
// combination applied. Every stage also reads the step-start state Q.
struct StagePlan {
    int n;
    int in[4], out[4], combo[4];
};

inline StagePlan plan_for(int stepper) {
    switch (stepper) {
        case 0:  // rk2
            return {2, {0, 1}, {1, 0}, {kAdd, kRk2Final}};
        case 1:  // ssprk3
            return {3, {0, 1, 2}, {1, 2, 0}, {kAdd, kSsp3Second, kSsp3Final}};
        default:  // ssprk4
            return {4, {0, 1, 2, 1}, {1, 2, 1, 0}, {kHalfAdd, kHalfAdd, kSsp4Third, kHalfAdd}};
    }
}

// One stage of an SSPRK step. pass selects, in 3D, the x-y plane pass (0)
// or the z pass that finishes the stage (1); in 2D, the stage (0) or the
// finishing (2) of a stage whose deferred-form tiles wrote only their
// divergence into p.dqxy; it is ignored in 1D.
cudaError_t launch_stage_d1_fp64(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d2_fp64(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d3_fp64(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d1_fp32(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d2_fp32(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d3_fp32(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
// The same with the gravity source term (p.gravity set).
cudaError_t launch_stage_d1_fp64_src(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d2_fp64_src(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d3_fp64_src(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d1_fp32_src(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d2_fp32_src(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d3_fp32_src(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
// 2D, the deferred form of the stage (pass 0 only): the tiles write their x+y
// divergence into p.dqxy, and pass 2 of the regular launcher finishes it.
cudaError_t launch_stage_d2_fp64_defer(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d2_fp32_defer(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d2_fp64_src_defer(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);
cudaError_t launch_stage_d2_fp32_src_defer(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s);

// Ghost fill of Q from its interior (every built-in boundary kind).
cudaError_t launch_fill_bcs(const StageParams& p, int ndim, cudaStream_t s);
// Primitives of p.q_in over every cell (ghosts included) into w, tracers
// as mass fractions.
cudaError_t launch_cons_to_prim(const StageParams& p, double* w, int ndim, cudaStream_t s);
// CFL minimum over every cell of Q (ghosts included) into blk->cfl_min_bits,
// which the launch first resets.
cudaError_t launch_cfl_min(const StageParams& p, int ndim, cudaStream_t s);
// CFL minimum over the ghost layers of the faces in face_mask (bit f = face
// f), folded into blk->cfl_min_bits without a reset.
cudaError_t launch_cfl_min_ghosts(const StageParams& p, int ndim, int face_mask, cudaStream_t s);
// Device-driven loop bookkeeping (see util_kernels.cu).
cudaError_t launch_clock_init(DeviceBlock* blk, double time, double max_time, double prev_output_time,
                              double output_delta, double max_cfl, cudaStream_t s);
cudaError_t launch_clock_advance(DeviceBlock* blk, double* dt_log, int first, cudaStream_t s);

// Record the message mc_last_error returns on this thread (capi.cu).
void set_last_error(const char* msg);

// Discrete adjoint, bit-exact parts (adjoint_exact.cu): the recording clock
// of the forward run (dt, CFL minimum, clamp flag of step `step`) and the
// search for the interior cell whose CFL bound equals *m_rec (into *idx).
cudaError_t launch_record_clock(DeviceBlock* blk, int first, double* dts, double* mins, int* clamped,
                                long long step, cudaStream_t s);
cudaError_t launch_cfl_argmin(const double* q, int nx, int ny, int ng, int xc, int yc, double gamma, double dx,
                              const double* m_rec, int* idx, cudaStream_t s);

} // namespace mc
