// Tangent-linear (forward-mode) derivative of n steps of the 2D scheme the
// discrete adjoint covers (WENO5-Z + HLLC, FP64, periodic faces; any SSPRK
// driver): mc_tangent_linear.
//
// The derivative is taken by evaluating the forward arithmetic of
// physics.cuh (cons_to_prim, WENO5-Z, HLLC, the CFL bound) and the stage
// combination of common.cuh on dual numbers: a value and N directional
// derivatives. The value part of every operation is the forward operation
// itself, compiled without contraction (-fmad=false), so it is bit-identical
// to the fused stage kernels and every branch (limiters, WENO weights, HLLC
// wave speeds, min / max / |x|) is taken as the forward run takes it; the
// derivative parts follow the chain rule on that branch. This makes the
// result an independent check of the hand-derived reverse sweep
// (adjoint_fma.cu): the two share the forward's branch choices and nothing
// else.
//
// Layout: one thread per interior cell evaluates its four faces (each face's
// two reconstructions from the primitives of the cells around it, no shared
// memory), so each face is solved twice and each cell reconstructed three
// times per axis. This is test-reference code, sized for grids like the
// adjoint's 512^2; it is not a tuned kernel.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "launch.h"
#include "mosscap_b200.h"

namespace mc {

// A value and N directional derivatives.
template <int N>
struct Dual {
    double v;
    double d[N];
    __device__ __forceinline__ Dual() : v(0.0) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            d[k] = 0.0;
        }
    }
    // constants (and forward values) carry no derivative
    __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            d[k] = 0.0;
        }
    }
    __device__ __forceinline__ Dual& operator+=(const Dual& b) {
        *this = *this + b;
        return *this;
    }
    __device__ __forceinline__ Dual& operator*=(const Dual& b) {
        *this = *this * b;
        return *this;
    }
    friend __device__ __forceinline__ Dual operator+(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v + b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = a.d[k] + b.d[k];
        }
        return r;
    }
    friend __device__ __forceinline__ Dual operator-(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v - b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = a.d[k] - b.d[k];
        }
        return r;
    }
    friend __device__ __forceinline__ Dual operator-(const Dual& a) {
        Dual r;
        r.v = -a.v;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = -a.d[k];
        }
        return r;
    }
    friend __device__ __forceinline__ Dual operator*(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v * b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = a.d[k] * b.v + a.v * b.d[k];
        }
        return r;
    }
    // (a / b)' = (a' - (a / b) b') / b
    friend __device__ __forceinline__ Dual operator/(const Dual& a, const Dual& b) {
        Dual r;
        r.v = a.v / b.v;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
        }
        return r;
    }
    friend __device__ __forceinline__ bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
    friend __device__ __forceinline__ bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
    friend __device__ __forceinline__ bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
    friend __device__ __forceinline__ bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
    // sqrt(x)' = x' / (2 sqrt(x))
    friend __device__ __forceinline__ Dual sqrt(const Dual& a) {
        Dual r;
        r.v = ::sqrt(a.v);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = a.d[k] / (2.0 * r.v);
        }
        return r;
    }
    // |x|' = sign(x) x', with sign(0) = 0 at the kink (the convention of the
    // reverse sweep, which takes the same zero subgradient there)
    friend __device__ __forceinline__ Dual fabs(const Dual& a) {
        Dual r;
        r.v = ::fabs(a.v);
        const double sg = a.v > 0.0 ? 1.0 : (a.v < 0.0 ? -1.0 : 0.0);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = sg * a.d[k];
        }
        return r;
    }
    // copysign(m, x) with a constant magnitude: piecewise constant
    friend __device__ __forceinline__ Dual copysign(const Dual& m, const Dual& x) {
        Dual r;
        r.v = ::copysign(m.v, x.v);
        const bool flip = signbit(m.v) != signbit(x.v);
#pragma unroll
        for (int k = 0; k < N; ++k) {
            r.d[k] = flip ? -m.d[k] : m.d[k];
        }
        return r;
    }
};

template <int N>
struct Consts<Dual<N>> {
    static constexpr double weno_eps = Consts<double>::weno_eps;
};

namespace {

constexpr int kDirs = 4;  // directions carried per pass
using D = Dual<kDirs>;
constexpr int kNv = 4;    // 2D hydro variables

struct TlmParams {
    const double* q_in;    // [4][yc][xc]
    const double* dq_in;   // [kDirs][4][yc][xc]
    const double* q_old;
    const double* dq_old;
    double* q_out;
    double* dq_out;
    int xc, yc, ng, nx, ny;
    long long plane;       // xc * yc
    double dx, gamma;
    const double* dgamma;  // [kDirs]
    const double* dt;      // [1 + kDirs]: the value and the derivatives of this step's dt
    int combo;
};

__device__ __forceinline__ D gamma_of(const TlmParams& p) {
    D g(p.gamma);
#pragma unroll
    for (int k = 0; k < kDirs; ++k) {
        g.d[k] = p.dgamma[k];
    }
    return g;
}

__device__ __forceinline__ void load_cell(const double* q, const double* dq, long long plane, long long c, D* out) {
#pragma unroll
    for (int v = 0; v < kNv; ++v) {
        out[v] = D(q[v * plane + c]);
#pragma unroll
        for (int k = 0; k < kDirs; ++k) {
            out[v].d[k] = dq[(k * kNv + v) * plane + c];
        }
    }
}

// primitives of the cell at array index (j, i)
__device__ __forceinline__ void prim_at(const TlmParams& p, const D& g, int j, int i, D* w) {
    D q[kNv];
    load_cell(p.q_in, p.dq_in, p.plane, (long long)j * p.xc + i, q);
    prim_from_cons<2>(g, q, w);
}

// One stage: the flux divergence of every interior cell and the stage
// combination, as the fused kernel forms them (integrate_flux,
// source/TimeStepping.cpp:10-35: (0 + dFx) + dFy, times dt / dx).
__global__ void __launch_bounds__(128) tlm_stage_kernel(TlmParams p) {
    const long long n = (long long)p.nx * p.ny;
    const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (c >= n) {
        return;
    }
    const int i = p.ng + (int)(c % p.nx);
    const int j = p.ng + (int)(c / p.nx);
    const D g = gamma_of(p);
    const D gfac = (g + D(1.0)) / (D(2.0) * g);
    D div[kNv];
#pragma unroll
    for (int v = 0; v < kNv; ++v) {
        div[v] = D(0.0);
    }
#pragma unroll 1
    for (int axis = 0; axis < 2; ++axis) {
        // primitives of the cells -3..+3 along the axis
        D w[7][kNv];
#pragma unroll
        for (int o = -3; o <= 3; ++o) {
            prim_at(p, g, axis == 0 ? j : j + o, axis == 0 ? i + o : i, w[o + 3]);
        }
        // face values: wr of cell -1, wl and wr of the cell, wl of cell +1
        D wr_m[kNv], wl_c[kNv], wr_c[kNv], wl_p[kNv];
#pragma unroll
        for (int v = 0; v < kNv; ++v) {
            D s[5], dummy;
#pragma unroll
            for (int o = 0; o < 5; ++o) {
                s[o] = w[o][v];
            }
            reconstruct<kWeno5z, kMonotonizedCentral>(s, dummy, wr_m[v]);
#pragma unroll
            for (int o = 0; o < 5; ++o) {
                s[o] = w[o + 1][v];
            }
            reconstruct<kWeno5z, kMonotonizedCentral>(s, wl_c[v], wr_c[v]);
#pragma unroll
            for (int o = 0; o < 5; ++o) {
                s[o] = w[o + 2][v];
            }
            reconstruct<kWeno5z, kMonotonizedCentral>(s, wl_p[v], dummy);
        }
        D f_lo[kNv], f_hi[kNv];
        riemann<kHllc, 2>(g, gfac, axis, wr_m, wl_c, f_lo);
        riemann<kHllc, 2>(g, gfac, axis, wr_c, wl_p, f_hi);
#pragma unroll
        for (int v = 0; v < kNv; ++v) {
            div[v] += f_lo[v] - f_hi[v];
        }
    }
    D dt(p.dt[0]);
#pragma unroll
    for (int k = 0; k < kDirs; ++k) {
        dt.d[k] = p.dt[1 + k];
    }
    const D dtdx = dt / D(p.dx);
    const D sdt = D(0.0) * dt;  // no source term
    const long long cell = (long long)j * p.xc + i;
    D qi[kNv], qo[kNv];
    load_cell(p.q_in, p.dq_in, p.plane, cell, qi);
    const bool old = combo_reads_old(p.combo);
    if (old) {
        load_cell(p.q_old, p.dq_old, p.plane, cell, qo);
    }
#pragma unroll
    for (int v = 0; v < kNv; ++v) {
        D qu = div[v];
        qu *= dtdx;
        const D r = combine<D>(p.combo, old ? qo[v] : D(0.0), qi[v], qu, sdt);
        p.q_out[v * p.plane + cell] = r.v;
#pragma unroll
        for (int k = 0; k < kDirs; ++k) {
            p.dq_out[(k * kNv + v) * p.plane + cell] = r.d[k];
        }
    }
}

// Periodic ghost fill of the value and the derivatives (every transform of
// a periodic face is the identity, so each ghost is a copy of its source).
__global__ void tlm_periodic_kernel(double* q, double* dq, int xc, int yc, int ng, int nx, int ny) {
    const long long plane = (long long)xc * yc;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < plane;
         c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % xc), j = (int)(c / xc);
        const bool gi = i < ng || i >= ng + nx, gj = j < ng || j >= ng + ny;
        if (!gi && !gj) {
            continue;
        }
        const int si = ng + (((i - ng) % nx) + nx) % nx;
        const int sj = ng + (((j - ng) % ny) + ny) % ny;
        const long long s = (long long)sj * xc + si;
        for (int v = 0; v < kNv; ++v) {
            q[v * plane + c] = q[v * plane + s];
            for (int k = 0; k < kDirs; ++k) {
                dq[(k * kNv + v) * plane + c] = dq[(k * kNv + v) * plane + s];
            }
        }
    }
}

// CFL minimum over the interior (periodic ghosts repeat it) into *bits.
__global__ void tlm_cfl_min_kernel(const double* q, int xc, int ng, int nx, int ny, double gamma, double dx,
                                   unsigned long long* bits) {
    const long long n = (long long)nx * ny;
    const long long plane = (long long)xc * (ny + 2 * ng);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const long long cell = (long long)(ng + c / nx) * xc + ng + c % nx;
        double qq[kNv], w[kNv];
#pragma unroll
        for (int v = 0; v < kNv; ++v) {
            qq[v] = q[v * plane + cell];
        }
        prim_from_cons<2>(gamma, qq, w);
        atomicMin(bits, ordered_bits(cfl_dt<2>(gamma, dx, w)));
    }
}

// The lowest interior index whose CFL bound equals the minimum.
__global__ void tlm_argmin_kernel(const double* q, int xc, int ng, int nx, int ny, double gamma, double dx,
                                  const unsigned long long* bits, int* idx) {
    const long long n = (long long)nx * ny;
    const long long plane = (long long)xc * (ny + 2 * ng);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < n;
         c += (long long)gridDim.x * blockDim.x) {
        const long long cell = (long long)(ng + c / nx) * xc + ng + c % nx;
        double qq[kNv], w[kNv];
#pragma unroll
        for (int v = 0; v < kNv; ++v) {
            qq[v] = q[v * plane + cell];
        }
        prim_from_cons<2>(gamma, qq, w);
        if (ordered_bits(cfl_dt<2>(gamma, dx, w)) == *bits) {
            atomicMin(idx, (int)c);
        }
    }
}

struct TlmClock {
    unsigned long long bits;
    int idx;
    double time, prev_output_time, max_time, output_delta, max_cfl;
    int steps, clamped;
    unsigned status;
};

__global__ void tlm_reset_kernel(TlmClock* k) {
    k->bits = kInfBits;
    k->idx = 0x7fffffff;
}

// dt = max_cfl * (CFL bound of the arg-min cell) with its derivative, then
// the output-time clamp of compute_dt (source/Hydro.cpp:231-241), which
// fixes dt (derivative zero). `close` first closes the previous step
// (time += dt; prev_output_time = time when an output fell due).
__global__ void tlm_clock_kernel(const double* q, const double* dq, int xc, int ng, int nx, int ny, double gamma,
                                 const double* dgamma, double dx, TlmClock* k, double* dt, int close) {
    if (close) {
        k->time += dt[0];
        k->steps += 1;
        if (k->time >= k->prev_output_time + k->output_delta) {
            k->prev_output_time = k->time;
        }
    }
    const long long plane = (long long)xc * (ny + 2 * ng);
    const int c = k->idx;
    if (c == 0x7fffffff) {
        k->status |= 0x8u;
        dt[0] = 0.0;
        for (int d = 0; d < kDirs; ++d) {
            dt[1 + d] = 0.0;
        }
        return;
    }
    const long long cell = (long long)(ng + c / nx) * xc + ng + c % nx;
    D g(gamma);
#pragma unroll
    for (int d = 0; d < kDirs; ++d) {
        g.d[d] = dgamma[d];
    }
    D qq[kNv], w[kNv];
    load_cell(q, dq, plane, cell, qq);
    prim_from_cons<2>(g, qq, w);
    const D m = cfl_dt<2>(g, D(dx), w);
    D t = m * D(k->max_cfl);
    const double next_write = smin(k->max_time, k->prev_output_time + k->output_delta);
    double v = t.v;
    k->clamped = 0;
    if (k->time + v >= next_write) {
        v = next_write - k->time;
        while (k->time + v < next_write) {
            v = nextafter(v, 1.7976931348623157e308);
        }
        t = D(v);
        k->clamped = 1;
    }
    dt[0] = t.v;
    for (int d = 0; d < kDirs; ++d) {
        dt[1 + d] = t.d[d];
    }
    if (!(t.v > 0.0) || !isfinite(t.v)) {
        k->status |= 0x8u;
    }
}

thread_local std::string g_msg;

mc_status tfail(mc_status s, const char* msg) {
    set_last_error(msg);
    return s;
}

mc_status tcuda(cudaError_t e, const char* where) {
    g_msg = std::string(where) + ": " + cudaGetErrorString(e);
    set_last_error(g_msg.c_str());
    return MC_ERR_CUDA;
}

} // namespace
} // namespace mc

extern "C" {

mc_status mc_tangent_linear(const mc_grid* grid, const mc_scheme* scheme, double* Q, double* dQ,
                            const double* dgamma, int32_t n_dirs, mc_clock* clock, int64_t n_steps, void* stream) {
    using namespace mc;
    if (!grid || !scheme || !Q || !dQ || !dgamma || !clock || n_dirs < 1 || n_steps < 0) {
        return tfail(MC_ERR_INVALID_ARGUMENT, "null argument, n_dirs < 1 or n_steps < 0");
    }
    const mc_grid& g = *grid;
    const mc_scheme& s = *scheme;
    if (g.num_dim != 2 || g.num_tracers != 0 || s.reconstruction != MC_RECON_WENO5Z ||
        s.riemann_solver != MC_RIEMANN_HLLC || s.precision != MC_PRECISION_FP64 || g.ng < 3 ||
        s.time_stepper < 0 || s.time_stepper > 2) {
        return tfail(MC_ERR_UNSUPPORTED, "the tangent-linear model covers the adjoint's scheme: 2D, WENO5-Z + HLLC, "
                                         "FP64, no tracers");
    }
    for (int f = 0; f < 4; ++f) {
        if (g.bc[f] != MC_BC_PERIODIC) {
            return tfail(MC_ERR_UNSUPPORTED, "the tangent-linear model needs periodic faces");
        }
    }
    const int nx = g.xc - 2 * g.ng, ny = g.yc - 2 * g.ng;
    if (nx < g.ng || ny < g.ng || g.zc != 1 || !(g.dx > 0.0)) {
        return tfail(MC_ERR_INVALID_ARGUMENT, "bad extents");
    }
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long plane = (long long)g.xc * g.yc;
    const size_t qn = size_t(kNv) * size_t(plane);
    const size_t dqn = size_t(kDirs) * qn;
    // device scratch: Q and stage buffers A, B (value and derivatives), the
    // step-start copy of Q, dgamma, dt and the clock
    std::vector<void*> owned;
    auto alloc = [&](void** p, size_t bytes) -> cudaError_t {
        const cudaError_t e = cudaMalloc(p, bytes);
        if (e == cudaSuccess) {
            owned.push_back(*p);
        }
        return e;
    };
    auto release = [&]() {
        for (void* p : owned) {
            cudaFree(p);
        }
        owned.clear();
    };
    double *q[3], *dq[3], *q0, *dq0, *dg, *dtv;
    TlmClock* kc;
    cudaError_t e = cudaSuccess;
    for (int b = 0; b < 3 && e == cudaSuccess; ++b) {
        e = alloc((void**)&q[b], qn * 8);
        if (e == cudaSuccess) {
            e = alloc((void**)&dq[b], dqn * 8);
        }
    }
    if (e == cudaSuccess) e = alloc((void**)&q0, qn * 8);
    if (e == cudaSuccess) e = alloc((void**)&dq0, dqn * 8);
    if (e == cudaSuccess) e = alloc((void**)&dg, kDirs * 8);
    if (e == cudaSuccess) e = alloc((void**)&dtv, (1 + kDirs) * 8);
    if (e == cudaSuccess) e = alloc((void**)&kc, sizeof(TlmClock));
    if (e != cudaSuccess) {
        release();
        return e == cudaErrorMemoryAllocation ? tfail(MC_ERR_OUT_OF_MEMORY, "device allocation") : tcuda(e, "alloc");
    }
    const StagePlan plan = plan_for(s.time_stepper);
    const int threads = 128;
    const int blocks = (int)(((long long)nx * ny + threads - 1) / threads);
    TlmClock host_clock{};
    mc_status status = MC_OK;
    for (int d0 = 0; d0 < n_dirs && status == MC_OK; d0 += kDirs) {
        const int nd = n_dirs - d0 < kDirs ? n_dirs - d0 : kDirs;
        // this pass's directions; unused slots stay zero
#define TL(call)                               \
    do {                                       \
        e = (call);                            \
        if (e != cudaSuccess) {                \
            status = tcuda(e, #call);          \
            break;                             \
        }                                      \
    } while (0)
        do {
            TL(cudaMemcpyAsync(q[0], Q, qn * 8, cudaMemcpyDefault, st));
            TL(cudaMemsetAsync(dq[0], 0, dqn * 8, st));
            TL(cudaMemcpyAsync(dq[0], dQ + size_t(d0) * qn, size_t(nd) * qn * 8, cudaMemcpyDefault, st));
            double dgh[kDirs] = {0.0, 0.0, 0.0, 0.0};
            for (int k = 0; k < nd; ++k) {
                dgh[k] = dgamma[d0 + k];
            }
            TL(cudaMemcpyAsync(dg, dgh, sizeof(dgh), cudaMemcpyHostToDevice, st));
            TlmClock k0{};
            k0.time = clock->time;
            k0.prev_output_time = clock->prev_output_time;
            k0.max_time = clock->max_time;
            k0.output_delta = clock->output_delta;
            k0.max_cfl = s.max_cfl;
            TL(cudaMemcpyAsync(kc, &k0, sizeof(k0), cudaMemcpyHostToDevice, st));
            TL(cudaStreamSynchronize(st));  // dgh and k0 live on this stack frame
            tlm_periodic_kernel<<<148, 256, 0, st>>>(q[0], dq[0], g.xc, g.yc, g.ng, nx, ny);
            tlm_reset_kernel<<<1, 1, 0, st>>>(kc);
            tlm_cfl_min_kernel<<<148 * 4, 256, 0, st>>>(q[0], g.xc, g.ng, nx, ny, s.gamma, g.dx, &kc->bits);
            tlm_argmin_kernel<<<148 * 4, 256, 0, st>>>(q[0], g.xc, g.ng, nx, ny, s.gamma, g.dx, &kc->bits, &kc->idx);
            tlm_clock_kernel<<<1, 1, 0, st>>>(q[0], dq[0], g.xc, g.ng, nx, ny, s.gamma, dg, g.dx, kc, dtv, 0);
            TL(cudaGetLastError());
            for (int64_t step = 0; step < n_steps && status == MC_OK; ++step) {
                TL(cudaMemcpyAsync(q0, q[0], qn * 8, cudaMemcpyDeviceToDevice, st));
                TL(cudaMemcpyAsync(dq0, dq[0], dqn * 8, cudaMemcpyDeviceToDevice, st));
                for (int k = 0; k < plan.n; ++k) {
                    TlmParams p;
                    std::memset(&p, 0, sizeof(p));
                    p.q_in = q[plan.in[k]];
                    p.dq_in = dq[plan.in[k]];
                    p.q_old = q0;
                    p.dq_old = dq0;
                    p.q_out = q[plan.out[k]];
                    p.dq_out = dq[plan.out[k]];
                    p.xc = g.xc;
                    p.yc = g.yc;
                    p.ng = g.ng;
                    p.nx = nx;
                    p.ny = ny;
                    p.plane = plane;
                    p.dx = g.dx;
                    p.gamma = s.gamma;
                    p.dgamma = dg;
                    p.dt = dtv;
                    p.combo = plan.combo[k];
                    tlm_stage_kernel<<<blocks, threads, 0, st>>>(p);
                    tlm_periodic_kernel<<<148, 256, 0, st>>>(q[plan.out[k]], dq[plan.out[k]], g.xc, g.yc, g.ng, nx,
                                                             ny);
                }
                tlm_reset_kernel<<<1, 1, 0, st>>>(kc);
                tlm_cfl_min_kernel<<<148 * 4, 256, 0, st>>>(q[0], g.xc, g.ng, nx, ny, s.gamma, g.dx, &kc->bits);
                tlm_argmin_kernel<<<148 * 4, 256, 0, st>>>(q[0], g.xc, g.ng, nx, ny, s.gamma, g.dx, &kc->bits,
                                                           &kc->idx);
                tlm_clock_kernel<<<1, 1, 0, st>>>(q[0], dq[0], g.xc, g.ng, nx, ny, s.gamma, dg, g.dx, kc, dtv, 1);
                TL(cudaGetLastError());
            }
            if (status != MC_OK) {
                break;
            }
            TL(cudaMemcpyAsync(dQ + size_t(d0) * qn, dq[0], size_t(nd) * qn * 8, cudaMemcpyDefault, st));
            if (d0 + kDirs >= n_dirs) {
                TL(cudaMemcpyAsync(Q, q[0], qn * 8, cudaMemcpyDefault, st));
            }
            TL(cudaMemcpyAsync(&host_clock, kc, sizeof(host_clock), cudaMemcpyDeviceToHost, st));
            TL(cudaStreamSynchronize(st));
        } while (0);
#undef TL
    }
    release();
    if (status != MC_OK) {
        return status;
    }
    clock->time = host_clock.time;
    clock->prev_output_time = host_clock.prev_output_time;
    if (host_clock.status) {
        return tfail(MC_ERR_STATE, "dt <= 0 or not finite in the tangent-linear run");
    }
    return MC_OK;
}

} // extern "C"
