// Batched stage kernel: one persistent launch advances one SSPRK stage of
// every problem of a batch of independent 1D and 2D problems of uneven size.
//
// The work list holds 2D tiles (one CTA each, the tile2d body of the single
// problem kernel) followed by bundles of kWarps 1D tasks (one warp each, a
// task being `nseg` consecutive 30-cell segments of one 1D problem, the
// segment1d body), so the warps of one CTA may serve different small
// problems. CTAs take work items either statically (item = blockIdx.x +
// k * gridDim.x) or dynamically from an atomic counter; the autotuner picks.
// Every problem has its own DeviceBlock: its dt, clock, CFL-minimum cell and
// status, so each problem advances with its own dt.
#pragma once

#include "stage_kernels.cuh"

namespace mc {

struct BatchItem2d {
    int prob, bx, by, pad;
};
struct BatchTask1d {
    int prob, s0, nseg, pad;  // segments s0 .. s0 + nseg - 1 of problem prob
};

struct BatchStageParams {
    const StageParams* probs;   // per-problem parameters (state pointers unset)
    const long long* offsets;   // per-problem offset into the state pools
    const BatchItem2d* items2d;
    int n2d;
    const BatchTask1d* tasks1d;
    int ntasks1d;
    int n_items;                // n2d + bundles of kWarps 1D tasks
    const double* in_base;      // pool of the stage input
    const double* old_base;     // pool of the step-start state
    double* out_base;           // pool of the stage output
    int combo;
    int last;
    int dynamic;
    int* counter;               // work counter of this launch (dynamic schedule)
};

template <int REC, class T>
__host__ __device__ constexpr size_t batch_smem_bytes() {
    // a 2D tile of 4 variables or kWarps 1D windows of 3 variables
    return smem_bytes<2, REC, T>(4) > smem_bytes<1, REC, T>(3) ? smem_bytes<2, REC, T>(4)
                                                               : smem_bytes<1, REC, T>(3);
}

__device__ __forceinline__ void bind_problem(StageParams& sp, const BatchStageParams& bp, int prob) {
    sp = bp.probs[prob];
    const long long off = bp.offsets[prob];
    sp.q_in = bp.in_base + off;
    sp.q_old = bp.old_base + off;
    sp.q_out = bp.out_base + off;
    sp.combo = bp.combo;
    sp.last = bp.last;
    sp.reset_min = 0;
}

template <int REC, int LIM, int RS, class T>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 4 ? kMinBlocks2dF32 : kMinBlocks2d)
    batch_stage_kernel(BatchStageParams bp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StageParams sp[kWarps];
    __shared__ double red_d[kWarps];
    __shared__ unsigned red_u[kWarps];
    __shared__ int s_item;
    T* smem = reinterpret_cast<T*>(smem_raw);
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    int item = blockIdx.x;
    for (;;) {
        if (bp.dynamic) {
            if (threadIdx.x == 0) {
                s_item = atomicAdd(bp.counter, 1);
            }
            __syncthreads();
            item = s_item;
        }
        if (item >= bp.n_items) {
            break;
        }
        if (item < bp.n2d) {
            const BatchItem2d it = bp.items2d[item];
            if (threadIdx.x == 0) {
                bind_problem(sp[0], bp, it.prob);
            }
            __syncthreads();
            if (!sp[0].blk->done) {
                double dtmin = __longlong_as_double((long long)kInfBits);
                unsigned flags = 0;
                tile2d<2, REC, LIM, RS, T>(sp[0], it.bx, it.by, 0, smem, dtmin, flags);
                block_publish(dtmin, flags, sp[0].last != 0, sp[0].blk, red_d, red_u);
            }
        } else {
            const int t = (item - bp.n2d) * kWarps + warp;
            if (t < bp.ntasks1d) {
                const BatchTask1d task = bp.tasks1d[t];
                if (lane == 0) {
                    bind_problem(sp[warp], bp, task.prob);
                }
                __syncwarp();
                const StageParams& p = sp[warp];
                if (!p.blk->done) {
                    double dtmin = __longlong_as_double((long long)kInfBits);
                    unsigned flags = 0;
                    T* W = smem + (size_t)warp * 3 * seg1d_window<REC>();
                    for (int s = 0; s < task.nseg; ++s) {
                        segment1d<REC, LIM, RS, T>(p, (task.s0 + s) * kTile, W, dtmin, flags);
                    }
                    dtmin = warp_min(dtmin);
                    flags = warp_or(flags);
                    if (lane == 0) {
                        if (p.last) {
                            atomicMin(&p.blk->cfl_min_bits, ordered_bits(dtmin));
                        }
                        if (flags) {
                            atomicOr(&p.blk->status, flags);
                        }
                    }
                }
            }
        }
        __syncthreads();
        if (!bp.dynamic) {
            item += gridDim.x;
        }
    }
}

} // namespace mc
