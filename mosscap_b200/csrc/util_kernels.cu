// Boundary fill, CFL reduction and the clock of the device-driven loop.
// Compiled with -fmad=false: the CFL bound and the dt clamp are bit-identical
// to the reference (source/Hydro.cpp:192-242).
#include <cuda_runtime.h>

#include "launch.h"
#include "stage_kernels.cuh"

namespace mc {

namespace {

inline int cdiv(long long a, long long b) {
    return (int)((a + b - 1) / b);
}

// fill_bcs (source/Boundaries.hpp:121-149) as a scatter: every interior
// cell that is the source of a ghost writes it (see write_cell). The
// interior is read and rewritten unchanged; ghosts are disjoint from it.
template <int NDIM>
__global__ void __launch_bounds__(256) fill_bcs_kernel(StageParams p) {
    const long long n = (long long)p.nx * p.ny * p.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const int xi = (int)(c % p.nx);
        const long long r = c / p.nx;
        const int yi = (int)(r % p.ny);
        const int zi = (int)(r / p.ny);
        const int i = xi + p.ng;
        const int j = NDIM > 1 ? yi + p.ng : 0;
        const int k = NDIM > 2 ? zi + p.ng : 0;
        const bool near = near_face(i, p.nx, p.ng) || (NDIM > 1 && near_face(j, p.ny, p.ng)) ||
                          (NDIM > 2 && near_face(k, p.nz, p.ng));
        if (!near) {
            continue;
        }
        double q[kMaxVars];
#pragma unroll
        for (int v = 0; v < kMaxVars; ++v) {
            q[v] = v < p.nvar ? p.q_out[qidx(p, v, k, j, i)] : 0.0;
        }
        unsigned flags = 0;
        write_cell<NDIM>(p, i, j, k, q, false, &flags);
    }
}

// dt_reducer over every cell, ghosts included (source/Hydro.cpp:209-229).
template <int NDIM>
__global__ void __launch_bounds__(256) cfl_min_kernel(StageParams p) {
    constexpr int nh = 2 + NDIM;
    __shared__ double red_d[8];
    __shared__ unsigned red_u[8];
    double m = __longlong_as_double((long long)kInfBits);
    unsigned flags = 0;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < p.plane;
         c += (long long)gridDim.x * blockDim.x) {
        double q[nh], w[nh];
        bool fin = true;
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            q[v] = p.q_in[v * p.plane + c];
            fin = fin && isfinite(q[v]);
        }
        prim_from_cons<NDIM>(p.gamma, q, w);
        flags |= state_flags(w[0], w[nh - 1], fin);
        m = smin(cfl_dt<NDIM>(p.gamma, p.dx, w), m);
    }
    block_publish(m, flags, true, p.blk, red_d, red_u);
}

// The CFL minimum over the ghost layers of the faces in face_mask (bit f =
// face f: xs, xe, ys, ye, zs, ze), whole extent along the other axes,
// folded into blk->cfl_min_bits without a reset. The fused stage kernels
// reduce over every value they write; the ghosts of MC_BC_USERFN faces are
// written afterwards by the caller's hook, and compute_dt reads every cell
// (source/Hydro.cpp:209-229), so those layers are added here.
template <int NDIM>
__global__ void __launch_bounds__(256) cfl_min_ghosts_kernel(StageParams p, int face_mask) {
    constexpr int nh = 2 + NDIM;
    __shared__ double red_d[8];
    __shared__ unsigned red_u[8];
    double m = __longlong_as_double((long long)kInfBits);
    unsigned flags = 0;
    const int ext[3] = {p.xc, p.yc, p.zc};
    for (int f = 0; f < 2 * NDIM; ++f) {
        if (!(face_mask & (1 << f))) {
            continue;
        }
        const int a = f >> 1;
        int lo[3] = {0, 0, 0}, n[3] = {ext[0], ext[1], ext[2]};
        lo[a] = (f & 1) ? ext[a] - p.ng : 0;
        n[a] = p.ng;
        const long long cells = (long long)n[0] * n[1] * n[2];
        for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < cells;
             c += (long long)gridDim.x * blockDim.x) {
            const int i = lo[0] + (int)(c % n[0]);
            const long long r = c / n[0];
            const int j = lo[1] + (int)(r % n[1]);
            const int k = lo[2] + (int)(r / n[1]);
            double q[nh], w[nh];
            bool fin = true;
#pragma unroll
            for (int v = 0; v < nh; ++v) {
                q[v] = p.q_in[qidx(p, v, k, j, i)];
                fin = fin && isfinite(q[v]);
            }
            prim_from_cons<NDIM>(p.gamma, q, w);
            flags |= state_flags(w[0], w[nh - 1], fin);
            m = smin(cfl_dt<NDIM>(p.gamma, p.dx, w), m);
        }
    }
    block_publish(m, flags, true, p.blk, red_d, red_u);
}

__global__ void reset_min_kernel(DeviceBlock* blk) {
    blk->cfl_min_bits = kInfBits;
}

__global__ void clock_init_kernel(DeviceBlock* blk, double time, double max_time, double prev_output_time,
                                  double output_delta, double max_cfl) {
    blk->cfl_min_bits = kInfBits;
    blk->dt = 0.0;
    blk->time = time;
    blk->max_time = max_time;
    blk->prev_output_time = prev_output_time;
    blk->output_delta = output_delta;
    blk->max_cfl = max_cfl;
    blk->steps = 0;
    blk->done = time < max_time ? 0 : 1;
}

__global__ void clock_advance_kernel(DeviceBlock* blk, double* dt_log, int first) {
    advance_clock(blk, dt_log, first != 0, true);
}

// global_cons_to_prim (source/Hydro.cpp:8-53) over every cell, ghosts
// included: the hydro primitives of q_in, and each tracer times 1 / rho.
template <int NDIM>
__global__ void __launch_bounds__(256) cons_to_prim_kernel(StageParams p, double* w_out) {
    constexpr int nh = 2 + NDIM;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < p.plane;
         c += (long long)gridDim.x * blockDim.x) {
        double q[nh], w[nh];
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            q[v] = p.q_in[v * p.plane + c];
        }
        prim_from_cons<NDIM>(p.gamma, q, w);
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            w_out[v * p.plane + c] = w[v];
        }
        if (p.ntracer > 0) {
            const double inv_rho = 1.0 / q[0];
            for (int t = 0; t < p.ntracer; ++t) {
                w_out[(nh + t) * p.plane + c] = p.q_in[(nh + t) * p.plane + c] * inv_rho;
            }
        }
    }
}

} // namespace

cudaError_t launch_cons_to_prim(const StageParams& p, double* w, int ndim, cudaStream_t s) {
    const int blocks = (int)(p.plane < 148LL * 8 * 256 ? cdiv(p.plane, 256) : 148 * 8);
    switch (ndim) {
        case 1:
            cons_to_prim_kernel<1><<<blocks, 256, 0, s>>>(p, w);
            break;
        case 2:
            cons_to_prim_kernel<2><<<blocks, 256, 0, s>>>(p, w);
            break;
        default:
            cons_to_prim_kernel<3><<<blocks, 256, 0, s>>>(p, w);
            break;
    }
    return cudaGetLastError();
}

cudaError_t launch_fill_bcs(const StageParams& p, int ndim, cudaStream_t s) {
    const long long n = (long long)p.nx * p.ny * p.nz;
    const int blocks = (int)(n < 148LL * 8 * 256 ? cdiv(n, 256) : 148 * 8);
    switch (ndim) {
        case 1:
            fill_bcs_kernel<1><<<blocks, 256, 0, s>>>(p);
            break;
        case 2:
            fill_bcs_kernel<2><<<blocks, 256, 0, s>>>(p);
            break;
        default:
            fill_bcs_kernel<3><<<blocks, 256, 0, s>>>(p);
            break;
    }
    return cudaGetLastError();
}

cudaError_t launch_cfl_min(const StageParams& p, int ndim, cudaStream_t s) {
    reset_min_kernel<<<1, 1, 0, s>>>(p.blk);
    const int blocks = (int)(p.plane < 148LL * 8 * 256 ? cdiv(p.plane, 256) : 148 * 8);
    switch (ndim) {
        case 1:
            cfl_min_kernel<1><<<blocks, 256, 0, s>>>(p);
            break;
        case 2:
            cfl_min_kernel<2><<<blocks, 256, 0, s>>>(p);
            break;
        default:
            cfl_min_kernel<3><<<blocks, 256, 0, s>>>(p);
            break;
    }
    return cudaGetLastError();
}

cudaError_t launch_cfl_min_ghosts(const StageParams& p, int ndim, int face_mask, cudaStream_t s) {
    const int blocks = 148;
    switch (ndim) {
        case 1:
            cfl_min_ghosts_kernel<1><<<blocks, 256, 0, s>>>(p, face_mask);
            break;
        case 2:
            cfl_min_ghosts_kernel<2><<<blocks, 256, 0, s>>>(p, face_mask);
            break;
        default:
            cfl_min_ghosts_kernel<3><<<blocks, 256, 0, s>>>(p, face_mask);
            break;
    }
    return cudaGetLastError();
}

cudaError_t launch_clock_init(DeviceBlock* blk, double time, double max_time, double prev_output_time,
                              double output_delta, double max_cfl, cudaStream_t s) {
    clock_init_kernel<<<1, 1, 0, s>>>(blk, time, max_time, prev_output_time, output_delta, max_cfl);
    return cudaGetLastError();
}

cudaError_t launch_clock_advance(DeviceBlock* blk, double* dt_log, int first, cudaStream_t s) {
    clock_advance_kernel<<<1, 1, 0, s>>>(blk, dt_log, first);
    return cudaGetLastError();
}

} // namespace mc
