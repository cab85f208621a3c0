// Kernels of the discrete adjoint that must reproduce forward values bit for
// bit (compiled with -fmad=false): the clock of the recorded forward run and
// the search for the cell whose CFL bound is the step's recorded minimum.
#include <cuda_runtime.h>

#include "launch.h"

namespace mc {

namespace {

// Forward clock of the recorded run: advance_clock without stopping at
// outputs, then record dt, the CFL minimum and whether the clamp fixed dt.
__global__ void record_clock_kernel(DeviceBlock* blk, int first, double* dts, double* mins, int* clamped,
                                    long long step) {
    advance_clock(blk, nullptr, first != 0, false);
    dts[step] = blk->dt;
    mins[step] = blk->last_cfl_min;
    clamped[step] = blk->dt != blk->last_cfl_min * blk->max_cfl;
}

__global__ void set_int_kernel(int* p, int v) {
    *p = v;
}

// The interior cell whose CFL bound (dt_reducer, source/Hydro.cpp:192-206)
// equals the recorded minimum, bit for bit (lowest index among exact ties).
// Periodic ghosts repeat interior values, so the interior holds the minimum.
__global__ void argmin_kernel(const double* q, int nx, int ny, int ng, int xc, int yc, double gamma, double dx,
                              const double* m_rec, int* idx) {
    const long long n = (long long)nx * ny;
    const unsigned long long target = (unsigned long long)__double_as_longlong(*m_rec);
    const long long plane = (long long)xc * yc;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x) {
        const int xi = (int)(c % nx), yi = (int)(c / nx);
        const long long cell = (long long)(yi + ng) * xc + xi + ng;
        double qq[4], w[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            qq[v] = q[v * plane + cell];
        }
        prim_from_cons<2>(gamma, qq, w);
        const double d = cfl_dt<2>(gamma, dx, w);
        if ((unsigned long long)__double_as_longlong(d) == target) {
            atomicMin(idx, (int)c);
        }
    }
}

} // namespace

cudaError_t launch_record_clock(DeviceBlock* blk, int first, double* dts, double* mins, int* clamped,
                                long long step, cudaStream_t s) {
    record_clock_kernel<<<1, 1, 0, s>>>(blk, first, dts, mins, clamped, step);
    return cudaGetLastError();
}

cudaError_t launch_cfl_argmin(const double* q, int nx, int ny, int ng, int xc, int yc, double gamma, double dx,
                              const double* m_rec, int* idx, cudaStream_t s) {
    set_int_kernel<<<1, 1, 0, s>>>(idx, 0x7fffffff);
    argmin_kernel<<<148 * 4, 256, 0, s>>>(q, nx, ny, ng, xc, yc, gamma, dx, m_rec, idx);
    return cudaGetLastError();
}

} // namespace mc
