// Batched stage kernels: persistent launches advance one SSPRK stage of
// every problem of a batch of independent 1D and 2D problems of uneven size.
//
// Two kinds of work item: a 2D tile (one CTA, the tile2d body of the
// single-problem kernel) and a bundle of 1D tasks, one per warp of the CTA
// (a task being `nseg` consecutive 30-cell segments of one 1D problem, the
// segment1d body), so the warps of one CTA may serve different small
// problems. PART kPartAll runs both in one persistent launch per stage: its
// work list is the 2D tiles, biggest problems first, then the 1D bundles.
// PARTs kPart2d and kPart1d split them into two launches, each kernel with
// the instruction footprint of one body; the autotuner picks the form. CTAs
// take work items either statically (item = blockIdx.x + k * gridDim.x) or
// dynamically from an atomic counter. Every problem has its own
// DeviceBlock: its dt, clock, CFL-minimum cell and status, so each problem
// advances with its own dt.
//
// Ghost cells: the work items store only their own cells. Each finished
// item is counted per problem (after a fence), and the CTA (2D) or warp
// (1D) that finishes a problem's last item of the stage fills that
// problem's ghost cells from the stored values (fill_ghosts). Nothing waits:
// the last finisher does the work. The values and CFL bounds are those of
// the single-problem kernels' per-cell scatter, without its divergence in
// the tile body (the scatter in the tile body took a quarter of the batch's
// time).
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
    // per-problem parameters of this stage (state pointers, combination and
    // last-stage flag bound), read in place from global memory
    const StageParams* probs;
    const BatchItem2d* items2d;
    int n2d;
    const BatchTask1d* tasks1d;
    int ntasks1d;
    int n_items;                // work items of this launch: the tiles, the 1D bundles or both
    int dynamic;
    int* counter;               // work counter of this launch (dynamic schedule)
    const int* items_of;        // per problem: its work items in a stage (2D tiles or 1D tasks)
    int* finished;              // per problem: its items of this stage finished so far
};

constexpr int kPart2d = 0;   // the launch over the 2D tiles
constexpr int kPart1d = 1;   // the launch over the 1D task bundles
constexpr int kPartAll = 2;  // one launch over both


// CTAs per SM of the batched kernels: the per-problem parameters come from
// global memory rather than the constant bank, so the tile body needs more
// registers than the single-problem kernel to keep them resident (two CTAs
// with up to 128 registers measured 7 % faster than three with 80).
constexpr int kMinBlocksBatch = 2;
// Threads per CTA: the 2D tiles run 320 (ten warps, three of a pass's 30
// lines each; 24 % faster than 256 on the 4096-problem set), so the merged
// kernel does too (bundles of ten 1D tasks); the 1D kernel alone runs one
// task per warp of 256.
template <int PART>
__host__ __device__ constexpr int batch_threads() {
    return PART == kPart1d ? kThreads : 320;
}
// 1D tasks per bundle: one per warp.
template <int PART>
__host__ __device__ constexpr int batch_warps() {
    return batch_threads<PART>() / 32;
}

template <int REC, class T, int PART>
__host__ __device__ constexpr size_t batch_smem_bytes() {
    // a 2D tile of 4 variables and / or one 1D window of 3 variables per warp
    constexpr size_t tile = smem_bytes<2, REC, T>(4);
    constexpr size_t windows = sizeof(T) * 3 * (size_t)batch_warps<PART>() * seg1d_window<REC>();
    return PART == kPart2d ? tile : PART == kPart1d ? windows : (tile > windows ? tile : windows);
}

template <int REC, int LIM, int RS, class T, int NT>
__device__ __forceinline__ void batch_tile(const BatchStageParams& bp, int item, T* smem, double* red_d,
                                           unsigned* red_u) {
    // the problem's parameters, bound to this stage's buffers, copied once
    // per tile into shared memory
    __shared__ StageParams s_p;
    const BatchItem2d it = bp.items2d[item];
    {
        const int* src = reinterpret_cast<const int*>(&bp.probs[it.prob]);
        int* dst = reinterpret_cast<int*>(&s_p);
        for (int k = threadIdx.x; k < (int)(sizeof(StageParams) / 4); k += NT) {
            dst[k] = src[k];
        }
    }
    __syncthreads();
    const StageParams& p = s_p;
    if (!p.blk->done) {
        double dtmin = __longlong_as_double((long long)kInfBits);
        unsigned flags = 0;
        tile2d<2, REC, LIM, RS, T, false, NT, false, false, false>(p, it.bx, it.by, 0, smem, dtmin, flags);
        block_publish(dtmin, flags, p.last != 0, p.blk, red_d, red_u);
        // the CTA that finishes the problem's last tile fills its ghost cells
        __shared__ int s_last;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            s_last = atomicAdd(&bp.finished[it.prob], 1) == bp.items_of[it.prob] - 1;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            unsigned gflags = 0;
            const double gmin = fill_ghosts<2, T>(p, threadIdx.x, NT, &gflags);
            block_publish(gmin, gflags, p.last != 0, p.blk, red_d, red_u);
        }
    }
}

template <int REC, int LIM, int RS, class T, int NW>
__device__ __forceinline__ void batch_bundle(const BatchStageParams& bp, int bundle, T* smem) {
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int t = bundle * NW + warp;
    if (t < bp.ntasks1d) {
        const BatchTask1d task = bp.tasks1d[t];
        const StageParams& p = bp.probs[task.prob];
        if (!p.blk->done) {
            double dtmin = __longlong_as_double((long long)kInfBits);
            unsigned flags = 0;
            T* W = smem + (size_t)warp * 3 * seg1d_window<REC>();
            for (int s = 0; s < task.nseg; ++s) {
                segment1d<REC, LIM, RS, T, false, false>(p, (task.s0 + s) * kTile, W, dtmin, flags);
            }
            // the warp that finishes the problem's last task fills its ghosts
            __threadfence();
            __syncwarp();
            int last = 0;
            if (lane == 0) {
                last = atomicAdd(&bp.finished[task.prob], 1) == bp.items_of[task.prob] - 1;
            }
            if (__shfl_sync(0xffffffffu, last, 0)) {
                __threadfence();
                dtmin = smin(fill_ghosts<1, T>(p, lane, 32, &flags), dtmin);
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

template <int REC, int LIM, int RS, class T, int PART>
__global__ void __launch_bounds__(batch_threads<PART>(), kMinBlocksBatch) batch_stage_kernel(BatchStageParams bp) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_d[batch_threads<PART>() / 32];
    __shared__ unsigned red_u[batch_threads<PART>() / 32];
    __shared__ int s_item;
    T* smem = reinterpret_cast<T*>(smem_raw);
    constexpr int NT = batch_threads<PART>();
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
        if constexpr (PART == kPart2d) {
            batch_tile<REC, LIM, RS, T, NT>(bp, item, smem, red_d, red_u);
        } else if constexpr (PART == kPart1d) {
            batch_bundle<REC, LIM, RS, T, batch_warps<PART>()>(bp, item, smem);
        } else if (item < bp.n2d) {
            batch_tile<REC, LIM, RS, T, NT>(bp, item, smem, red_d, red_u);
        } else {
            batch_bundle<REC, LIM, RS, T, batch_warps<PART>()>(bp, item - bp.n2d, smem);
        }
        __syncthreads();
        if (!bp.dynamic) {
            item += gridDim.x;
        }
    }
}

} // namespace mc
