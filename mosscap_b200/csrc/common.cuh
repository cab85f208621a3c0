// Shared device-side definitions of the Euler-step kernels: launch
// parameters, the device control block, SSPRK stage combinations, boundary
// transforms and the order-preserving CFL minimum.
#pragma once

#include <cstdint>

#include "physics.cuh"

namespace mc {

constexpr int kMaxVars = 8;   // 2 + num_dim hydro variables plus tracers
constexpr int kMaxGhost = 8;  // ghost cells per side accepted by the library

enum Bc : int { kWall = 0, kPeriodic, kSymmetric, kDiode, kZeroGrad, kConstant, kUserFn };

// Stage combinations of the SSPRK drivers (source/TimeStepping.cpp).
enum Combo : int {
    kAdd = 0,        // Q_in + (L + S)              rk2 0, ssprk3 0        :66, :143
    kRk2Final,       // 0.5 (Q_old + Q_in + L + S)  rk2 1                  :86
    kSsp3Second,     // 3/4 Q_old + 1/4 (Q_in + L + S)      ssprk3 1       :163
    kSsp3Final,      // 1/3 Q_old + 2/3 (Q_in + L + S)      ssprk3 2       :183
    kHalfAdd,        // Q_in + 1/2 (L + S)          ssprk4 0, 1, 3         :240, :260, :300
    kSsp4Third       // 2/3 Q_old + 1/3 Q_in + 1/6 (L + S)  ssprk4 2       :280
};

// Device control block: one per context, in device memory.
struct DeviceBlock {
    unsigned long long cfl_min_bits;  // atomicMin target: bits of a non-negative double
    double dt;                        // dt of the step in flight (device-driven loop)
    double time;
    double prev_output_time;
    double max_time;
    double output_delta;
    double max_cfl;
    double last_cfl_min;              // CFL minimum of the last completed step
    long long steps;                  // steps taken by the device-driven loop
    int done;                         // nonzero: the device-driven loop has stopped
    unsigned status;                  // MC_FLAG_* bits
};

struct BcDesc {
    int kind[6];            // xs, xe, ys, ye, zs, ze
    double cval[6][kMaxVars];
};

// Launch parameters of one stage.
struct StageParams {
    const double* __restrict__ q_in;  // stage input, ghosts filled
    const double* q_old;              // step-start state, read only at the written cell
    double* q_out;                    // stage output (interior and ghosts)
    double* dqxy;                     // 3D only: x+y flux divergence per interior cell
    int xc, yc, zc, ng;
    int nx, ny, nz;                   // interior extents
    int nvar, ntracer;
    long long plane;                  // xc * yc * zc
    double dx, gamma;
    double dt;                        // used when dt_dev is null
    const double* dt_dev;             // device dt (the device-driven loop)
    int combo;
    int last;                         // nonzero in the last stage: CFL minimum + checks
    int reset_min;                    // nonzero: reset blk->cfl_min_bits (a stage before the last)
    BcDesc bc;
    DeviceBlock* blk;
    int gravity;                      // nonzero: the gravity source term is registered
    double grav[3];                   // its acceleration (x, y, z)
    // 2D launches over some of the tile rows (the slab exchange's overlap):
    // tile row = blockIdx.y, plus row_skip from blockIdx.y = row_split on;
    // tile_rows, if nonzero, is the launch's grid height. All zero: every
    // tile row, one per blockIdx.y.
    int row_split, row_skip, tile_rows;
};

constexpr unsigned long long kInfBits = 0x7ff0000000000000ull;

// Output cells per warp-wide row segment: the side of a 2D tile and the
// length of a 1D segment or z column chunk.
constexpr int kTile = 30;

// Called at the top of every stage kernel: a stage that is not the last one
// clears the CFL-minimum cell that the last stage will reduce into.
__device__ __forceinline__ void maybe_reset_min(const StageParams& p) {
    if (p.reset_min && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0 && threadIdx.x == 0 &&
        threadIdx.y == 0 && threadIdx.z == 0) {
        p.blk->cfl_min_bits = kInfBits;
    }
}

__device__ __forceinline__ double stage_dt(const StageParams& p) {
    return p.dt_dev ? *p.dt_dev : p.dt;
}

// Source term times dt of the 2 + NDIM hydro variables of interior cell
// (k, j, i), evaluated from the stage input as the reference does: every
// stage zeroes S (source/SourceTerms.hpp:8-10) and the registered source
// terms then add to it from the current state (:12-16); the only source term
// of the reference, gravity (source/SourceTerms/Gravity.cpp:16-41), adds
// rho g_a to each momentum and m_x g_x (+ m_y g_y (+ m_z g_z)) to the energy;
// the stage update adds S dt (source/TimeStepping.cpp:60-66). SRC is false
// in the kernels launched without a source term: S stays 0 and the result is
// 0 * dt.
// This form takes the cell's stage-input state q[0..1+NDIM] from the caller.
template <int NDIM, bool SRC>
__device__ __forceinline__ void source_dt_of(const StageParams& p, const double* qc, double dt, double* sdt) {
    constexpr int nh = 2 + NDIM;
    if constexpr (!SRC) {
        (void)p;
        (void)qc;
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            sdt[v] = 0.0 * dt;
        }
        return;
    }
    auto q = [&](int v) { return qc[v]; };
    const double rho = q(0);
    double S[nh];
    S[0] = 0.0;
    double energy_update = q(1) * p.grav[0];
    S[1] = 0.0 + rho * p.grav[0];
    if constexpr (NDIM > 1) {
        S[2] = 0.0 + rho * p.grav[1];
        energy_update += q(2) * p.grav[1];
    }
    if constexpr (NDIM > 2) {
        S[3] = 0.0 + rho * p.grav[2];
        energy_update += q(3) * p.grav[2];
    }
    S[1 + NDIM] = 0.0 + energy_update;
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        sdt[v] = S[v] * dt;
    }
}

template <int NDIM, bool SRC>
__device__ __forceinline__ void source_dt(const StageParams& p, int k, int j, int i, double dt, double* sdt) {
    constexpr int nh = 2 + NDIM;
    double q[nh];
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        if constexpr (SRC) {
            q[v] = p.q_in[(((long long)v * p.zc + k) * p.yc + j) * (long long)p.xc + i];
        } else {
            q[v] = 0.0;
        }
    }
    source_dt_of<NDIM, SRC>(p, q, dt, sdt);
}

// One SSPRK stage update of one variable; qu is the flux divergence already
// multiplied by dt/dx and src the source term times dt. T is double in the
// stage kernels (and a dual number in the tangent-linear kernels).
template <class T>
__device__ __forceinline__ T combine(int combo, T q_old, T q_in, T qu, T src) {
    switch (combo) {
        case kAdd:
            return q_in + (qu + src);
        case kRk2Final:
            return T(0.5) * (q_old + q_in + qu + src);
        case kSsp3Second:
            return T(0.75) * q_old + T(0.25) * (q_in + qu + src);
        case kSsp3Final:
            return T(1.0 / 3.0) * q_old + T(2.0 / 3.0) * (q_in + qu + src);
        case kHalfAdd:
            return q_in + T(0.5) * (qu + src);
        default:
            return T(2.0 / 3.0) * q_old + T(1.0 / 3.0) * q_in + T(1.0 / 6.0) * (qu + src);
    }
}

// combine() over the first N variables with one dispatch on the combination
// (the same expression per variable).
template <int N>
__device__ __forceinline__ void combine_all(int combo, const double* q_old, const double* q_in, const double* qu,
                                            const double* src, double* out) {
    switch (combo) {
        case kAdd:
#pragma unroll
            for (int v = 0; v < N; ++v) {
                out[v] = combine(kAdd, q_old[v], q_in[v], qu[v], src[v]);
            }
            break;
        case kRk2Final:
#pragma unroll
            for (int v = 0; v < N; ++v) {
                out[v] = combine(kRk2Final, q_old[v], q_in[v], qu[v], src[v]);
            }
            break;
        case kSsp3Second:
#pragma unroll
            for (int v = 0; v < N; ++v) {
                out[v] = combine(kSsp3Second, q_old[v], q_in[v], qu[v], src[v]);
            }
            break;
        case kSsp3Final:
#pragma unroll
            for (int v = 0; v < N; ++v) {
                out[v] = combine(kSsp3Final, q_old[v], q_in[v], qu[v], src[v]);
            }
            break;
        case kHalfAdd:
#pragma unroll
            for (int v = 0; v < N; ++v) {
                out[v] = combine(kHalfAdd, q_old[v], q_in[v], qu[v], src[v]);
            }
            break;
        default:
#pragma unroll
            for (int v = 0; v < N; ++v) {
                out[v] = combine(kSsp4Third, q_old[v], q_in[v], qu[v], src[v]);
            }
            break;
    }
}

__host__ __device__ inline bool combo_reads_old(int combo) {
    return combo == kRk2Final || combo == kSsp3Second || combo == kSsp3Final || combo == kSsp4Third;
}

// ---- Boundary conditions as a scatter ----------------------------------------
//
// fill_bcs (source/Boundaries.hpp:11-149) fills x ghosts, then y ghosts over
// the full x extent, then z ghosts over the full x-y extent. Every ghost value
// it produces is a transform of one interior cell: ghost (gx, gy, gz) ends up
// as Tz(Ty(Tx(Q[sz][sy][sx]))), where along each axis s is the source index
// of the ghost (itself for interior indices) and T the face's transform
// (identity for interior indices). The kernels below therefore write, next to
// each interior cell they update, every ghost whose source it is.

// Ghost targets of array index c along one axis. Entry 0 is c itself
// (no transform). face[] is -1 for c itself, 0 for the start face, 1 for the
// end face. n interior cells, ng ghosts, requires n >= ng.
__device__ __forceinline__ int axis_targets(int c, int n, int ng, int bs, int be, int* idx, int* face) {
    int cnt = 0;
    idx[cnt] = c;
    face[cnt++] = -1;
    // start face: ghosts 0..ng-1
    if (bs == kPeriodic) {
        if (c >= n && c < n + ng) {  // ghost g takes g + n
            idx[cnt] = c - n;
            face[cnt++] = 0;
        }
    } else if (bs == kWall || bs == kSymmetric || bs == kDiode) {
        if (c >= ng && c < 2 * ng) {  // mirror about the face
            idx[cnt] = 2 * ng - 1 - c;
            face[cnt++] = 0;
        }
    } else if (bs == kZeroGrad || bs == kConstant) {
        if (c == ng) {
            for (int g = 0; g < ng; ++g) {
                idx[cnt] = g;
                face[cnt++] = 0;
            }
        }
    }
    // end face: ghosts ng+n .. 2ng+n-1
    if (be == kPeriodic) {
        if (c >= ng && c < 2 * ng) {
            idx[cnt] = c + n;
            face[cnt++] = 1;
        }
    } else if (be == kWall || be == kSymmetric || be == kDiode) {
        if (c >= n && c < n + ng) {
            idx[cnt] = 2 * (ng + n) - 1 - c;
            face[cnt++] = 1;
        }
    } else if (be == kZeroGrad || be == kConstant) {
        if (c == ng + n - 1) {
            for (int g = 0; g < ng; ++g) {
                idx[cnt] = ng + n + g;
                face[cnt++] = 1;
            }
        }
    }
    return cnt;
}

// The same targets one at a time, without arrays (so that a kernel keeps
// them in registers): the number of targets of index c (entry 0 is c
// itself) and target k with its face (-1 for c itself, 0 start, 1 end), in
// the order axis_targets lists them.
__device__ __forceinline__ int start_target_count(int c, int n, int ng, int bs) {
    if (bs == kPeriodic) {
        return (c >= n && c < n + ng) ? 1 : 0;
    }
    if (bs == kWall || bs == kSymmetric || bs == kDiode) {
        return (c >= ng && c < 2 * ng) ? 1 : 0;
    }
    if (bs == kZeroGrad || bs == kConstant) {
        return c == ng ? ng : 0;
    }
    return 0;
}
__device__ __forceinline__ int end_target_count(int c, int n, int ng, int be) {
    if (be == kPeriodic) {
        return (c >= ng && c < 2 * ng) ? 1 : 0;
    }
    if (be == kWall || be == kSymmetric || be == kDiode) {
        return (c >= n && c < n + ng) ? 1 : 0;
    }
    if (be == kZeroGrad || be == kConstant) {
        return c == ng + n - 1 ? ng : 0;
    }
    return 0;
}
__device__ __forceinline__ int axis_target_at(int c, int n, int ng, int bs, int be, int ns, int k, int* face) {
    if (k == 0) {
        *face = -1;
        return c;
    }
    k -= 1;
    if (k < ns) {
        *face = 0;
        if (bs == kPeriodic) {
            return c - n;
        }
        if (bs == kZeroGrad || bs == kConstant) {
            return k;
        }
        return 2 * ng - 1 - c;
    }
    k -= ns;
    *face = 1;
    if (be == kPeriodic) {
        return c + n;
    }
    if (be == kZeroGrad || be == kConstant) {
        return ng + n + k;
    }
    return 2 * (ng + n) - 1 - c;
}

// Whether array index c along an axis feeds any ghost (fast-path test).
__device__ __forceinline__ bool near_face(int c, int n, int ng) {
    return c < 2 * ng || c >= n;
}

// Apply the transform of face `face` (0 start, 1 end) of axis `axis`
// to a conserved vector                                   Boundaries.hpp:83-115
template <int NDIM>
__device__ __forceinline__ void bc_transform(const BcDesc& bc, int axis, int face, int nvar, double* q) {
    const int kind = bc.kind[2 * axis + face];
    const int im = 1 + axis;
    constexpr int ie = 1 + NDIM;
    if (kind == kWall) {
        q[im] = -q[im];
    } else if (kind == kDiode) {
        const double mom_pre = q[im];
        q[im] = face == 0 ? smin(mom_pre, 0.0) : smax(mom_pre, 0.0);
        q[ie] -= sq(q[im] - mom_pre) / q[0];
    } else if (kind == kConstant) {
#pragma unroll
        for (int v = 0; v < kMaxVars; ++v) {
            if (v < nvar) {
                q[v] = bc.cval[2 * axis + face][v];
            }
        }
    }
}

// ---- Status checks and the CFL minimum ----------------------------------------

__device__ __forceinline__ unsigned state_flags(double rho, double p, bool finite) {
    unsigned f = 0;
    if (!finite) {
        f |= 0x1u;
    }
    if (!(rho > 0.0)) {
        f |= 0x2u;
    }
    if (!(p > 0.0)) {
        f |= 0x4u;
    }
    return f;
}

// Non-negative doubles (and +inf) order like their bit patterns read as
// unsigned integers, so an integer atomicMin on the bits is an exact,
// order-independent floating-point minimum. NaN is mapped to +inf bits (and
// flagged separately).
__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    if (!(v == v)) {
        return 0x7ff0000000000000ull;
    }
    if (v <= 0.0) {
        return 0ull;
    }
    return static_cast<unsigned long long>(__double_as_longlong(v));
}

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v = smin(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

__device__ __forceinline__ unsigned warp_or(unsigned v) {
    return __reduce_or_sync(0xffffffffu, v);
}

// Block-wide min of v and OR of flags; thread 0 publishes both with one
// atomic each. red_d / red_u hold one entry per warp of the block.
__device__ __forceinline__ void block_publish(double v, unsigned flags, bool do_min, DeviceBlock* blk,
                                              double* red_d, unsigned* red_u) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nw = (blockDim.x * blockDim.y * blockDim.z) >> 5;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    v = warp_min(v);
    flags = warp_or(flags);
    if (lane == 0) {
        red_d[warp] = v;
        red_u[warp] = flags;
    }
    __syncthreads();
    if (tid == 0) {
        double m = red_d[0];
        unsigned f = red_u[0];
        for (int w = 1; w < nw; ++w) {
            m = smin(m, red_d[w]);
            f |= red_u[w];
        }
        if (do_min) {
            atomicMin(&blk->cfl_min_bits, ordered_bits(m));
        }
        if (f) {
            atomicOr(&blk->status, f);
        }
    }
}

// Close the step that just finished (unless `first`) and pick the next dt
// of one problem's clock:
//   time += dt; an output falls due when time >= prev_output_time + delta
//   (source/main.cpp:67-71), which sets prev_output_time = time
//   (source/Output.cpp:272); the loop ends once time >= max_time
//   (source/main.cpp:54), and, with stop_at_output, also after a step that
//   made an output due (so that the host can write it);
//   dt = max_cfl * min, clamped to end exactly on the next output time
//   (source/Hydro.cpp:231-241).
__device__ __forceinline__ void advance_clock(DeviceBlock* blk, double* dt_log, bool first, bool stop_at_output) {
    if (blk->done) {
        return;
    }
    const double m = __longlong_as_double((long long)blk->cfl_min_bits);
    blk->cfl_min_bits = kInfBits;
    blk->last_cfl_min = m;
    if (!first) {
        blk->time += blk->dt;
        blk->steps += 1;
        bool stop = false;
        if (blk->time >= blk->prev_output_time + blk->output_delta) {
            blk->prev_output_time = blk->time;
            stop = stop_at_output;
        }
        if (!(blk->time < blk->max_time)) {
            stop = true;
        }
        if (stop) {
            blk->done = 1;
            return;
        }
    }
    double dt = m * blk->max_cfl;
    const double next_write = smin(blk->max_time, blk->prev_output_time + blk->output_delta);
    if (blk->time + dt >= next_write) {
        dt = next_write - blk->time;
        while (blk->time + dt < next_write) {
            dt = nextafter(dt, 1.7976931348623157e308);
        }
    }
    blk->dt = dt;
    if (dt_log) {
        dt_log[blk->steps] = dt;
    }
    if (!(dt > 0.0) || !isfinite(dt)) {
        blk->status |= 0x8u;
        blk->done = 1;
    }
}

} // namespace mc
