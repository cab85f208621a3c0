// Discrete adjoint of the 2D Euler step (WENO5-Z + HLLC + SSPRK3, FP64,
// periodic faces): the exact vector-Jacobian product of the discrete map
// Q_n -> Q_{n+1} that the forward kernels compute, including the dependence
// of each step's dt on the state (the CFL minimum, through its arg-min
// cell) and the dependence on gamma.
//
// Forward (mc_adjoint_forward): the device-driven loop, recording every
// step's dt, CFL minimum and whether the output clamp fixed dt, and storing
// the state every `checkpoint_every` steps.
// Backward (mc_adjoint_backward): per checkpoint segment, last first, the
// segment's stage states are recomputed from its checkpoint with the forward
// kernels (bit-identical), then the steps are reversed stage by stage:
//   stage   Q_out = a Q_old + b (Q_in + dt L(Q_in))
//   adjoint lam_in  = b lam_out + b dt J_L(Q_in)^T lam_out
//           lam_old += a lam_out,  g_dt += b <lam_out, L(Q_in)>,
//           g_gamma += b dt <lam_out, dL/dgamma>
// and each step's g_dt flows back through dt = max_cfl * dx / (c_s + |v|)
// at the arg-min cell (unless the step's dt was clamped to an output time).
// Split into y slabs over ranks (mc_adjoint_set_slab_*), the forward and the
// recompute exchange ghost rows after every stage, and each stage's product
// reads the bordering rows of its input and cotangent from the neighbours
// (halo buffers) instead of wrapping around the slab.
// The reverse sweep's own arithmetic need not be bit-exact, so this unit is
// compiled with multiply-add contraction; the forward recompute (the stage
// kernels), the arg-min search and the recording clock run in units compiled
// without it (adjoint_exact.cu), so the recompute is bit-identical.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "adjoint_physics.cuh"
#include "launch.h"
#include "mosscap_b200.h"
#include "slab.h"

using mc::DeviceBlock;
using mc::StageParams;

namespace {

// The adjoint tile is AT x AT output cells. A warp sweeps one line of the
// tile with lane L on cell L - 3: cells -3 .. 28 are reconstructed, faces
// -2 .. AT are solved and the stencil cotangents of cells -2 .. AT + 1 are
// gathered into the AT own cells, so AT <= 26. kTile = 26 measured as fast
// as 24 on the 512^2 adjoint (24 gives every warp 3 lines per pass, 26
// gives two of the eight warps a fourth) with fewer halo cells per output.
constexpr int kTile = 26;
constexpr int kAH = 5;                // primitive halo (stencils of the reconstructions feeding the faces)
constexpr int kMH = 3;                // cotangent halo
constexpr int kAThreads = 256;
constexpr int kAWarps = kAThreads / 32;

template <int AT>
struct VjpTile {
    static constexpr int kAW = AT + 2 * kAH;  // stored rows / columns of primitives
    static constexpr int kAP = kAW + 1;       // odd pitch
    static constexpr int kMW = AT + 2 * kMH;  // stored rows / columns of cotangents
    static constexpr int kMP = kMW + 1;
    static constexpr int kBP = AT + 1;        // pitch of the tile's primitive cotangents
    static size_t smem_bytes() { return sizeof(double) * 4 * (size_t)(kAW * kAP + kMW * kMP + AT * kBP); }
};

struct VjpParams {
    const double* q;        // stage input (padded layout, periodic ghosts)
    const double* mu;       // cotangent of the stage output (interior cells used)
    double* lam;            // out: cotangent of the stage input (interior cells)
    const double* add;      // optional, added to lam
    const double* acc_in;   // optional accumulator of the step-start cotangent
    double* acc_out;        // optional: acc_out = acc_in + a * mu
    const double* dt;       // device dt of the step
    // Rows beyond the slab (slab decomposition; NULL: periodic wrap within
    // the grid): [4][kAH][xc] rows -kAH .. -1 and ny .. ny + kAH - 1 of the
    // stage input, [4][kMH][xc] the same of the cotangent.
    const double* qlo;
    const double* qhi;
    const double* mlo;
    const double* mhi;
    double a, b;
    double dx, gamma;
    int nx, ny, ng, xc, yc;
    double* part_gdt;       // per-CTA sum of <mu, divergence>
    double* part_gam;       // per-CTA gamma cotangent
};

__device__ __forceinline__ int wrap(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

__device__ __forceinline__ long long pidx(const VjpParams& p, int v, int j, int i) {
    return ((long long)v * p.yc + j) * (long long)p.xc + i;
}

// Variable v of the cell in padded column i and slab row gy (gy >= -H): own
// rows from the state, rows beyond the slab from the H-row halo of the
// neighbour (rows past the halo, which no own cell's result reads, repeat
// its last row), or without halos the periodic image.
__device__ __forceinline__ double slab_at(const VjpParams& p, const double* own, const double* lo, const double* hi,
                                          int H, int v, int gy, int i) {
    if (!lo) {
        return own[pidx(p, v, p.ng + wrap(gy, p.ny), i)];
    }
    if (gy < 0) {
        return lo[((long long)v * H + gy + H) * p.xc + i];
    }
    if (gy >= p.ny) {
        return hi[((long long)v * H + min(gy - p.ny, H - 1)) * p.xc + i];
    }
    return own[pidx(p, v, p.ng + gy, i)];
}

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[warp] = v;
    }
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < kAWarps; ++w) {
            s += red[w];
        }
    }
    __syncthreads();
    return s;
}

template <int AT>
__global__ void __launch_bounds__(kAThreads, 2) stage_vjp_kernel(VjpParams p) {
    using TL = VjpTile<AT>;
    constexpr int kAW = TL::kAW, kAP = TL::kAP, kMW = TL::kMW, kMP = TL::kMP, kBP = TL::kBP;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* W = reinterpret_cast<double*>(smem_raw);   // [4][kAW][kAP]
    double* MU = W + 4 * kAW * kAP;                     // [4][kMW][kMP]
    double* WB = MU + 4 * kMW * kMP;                    // [4][AT][kBP]
    __shared__ double red[kAWarps];
    const int x0 = blockIdx.x * AT, y0 = blockIdx.y * AT;
    const int vw = min(AT, p.nx - x0), vh = min(AT, p.ny - y0);
    const double gamma = p.gamma;
    const mc::GasK K = mc::gas_constants(gamma);

    // primitives with a periodic cross-shaped halo of kAH cells
    {
        constexpr int core = AT * kAW;
        constexpr int items = core + 2 * kAH * AT;
        for (int it = threadIdx.x; it < items; it += kAThreads) {
            int tx, ty;
            if (it < core) {
                ty = it / kAW;
                tx = it - ty * kAW - kAH;
            } else {
                const int r = it - core;
                const int hr = r / AT;
                tx = r - hr * AT;
                ty = hr < kAH ? hr - kAH : AT + hr - kAH;
            }
            const int i = p.ng + wrap(x0 + tx, p.nx);
            double q[4], w[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                q[v] = slab_at(p, p.q, p.qlo, p.qhi, kAH, v, y0 + ty, i);
            }
            mc::prim_from_cons_rev2(K.gm1, q, w);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                W[(v * kAW + ty + kAH) * kAP + tx + kAH] = w[v];
            }
        }
        constexpr int mcore = AT * kMW;
        constexpr int mitems = mcore + 2 * kMH * AT;
        for (int it = threadIdx.x; it < mitems; it += kAThreads) {
            int tx, ty;
            if (it < mcore) {
                ty = it / kMW;
                tx = it - ty * kMW - kMH;
            } else {
                const int r = it - mcore;
                const int hr = r / AT;
                tx = r - hr * AT;
                ty = hr < kMH ? hr - kMH : AT + hr - kMH;
            }
            const int i = p.ng + wrap(x0 + tx, p.nx);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                MU[(v * kMW + ty + kMH) * kMP + tx + kMH] = slab_at(p, p.mu, p.mlo, p.mhi, kMH, v, y0 + ty, i);
            }
        }
        for (int it = threadIdx.x; it < 4 * AT * kBP; it += kAThreads) {
            WB[it] = 0.0;
        }
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int r = lane - 3;  // this lane's cell along the sweep (-3 .. 28)
    const double s = p.b * (*p.dt) / p.dx;
    double gdt = 0.0, gam = 0.0;
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        const int axis = pass;  // rows (x faces) first, then columns (y faces)
        const int nlines = axis == 0 ? vh : vw;
        for (int line = warp; line < nlines; line += kAWarps) {
            // this lane's reconstruction stencils (4 variables x 5 points)
            auto wat = [&](int v, int o) -> double {
                return axis == 0 ? W[(v * kAW + line + kAH) * kAP + r + o + kAH]
                                 : W[(v * kAW + r + o + kAH) * kAP + line + kAH];
            };
            double rl[4], rr[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                double st[5];
#pragma unroll
                for (int o = 0; o < 5; ++o) {
                    st[o] = wat(v, o - 2);
                }
                mc::weno5z_faces(st, rl[v], rr[v]);
            }
            double left[4], mu_r[4], mu_l[4], fb[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                left[v] = __shfl_up_sync(0xffffffffu, rr[v], 1);
                mu_r[v] = axis == 0 ? MU[(v * kMW + line + kMH) * kMP + r + kMH]
                                    : MU[(v * kMW + r + kMH) * kMP + line + kMH];
                mu_l[v] = __shfl_up_sync(0xffffffffu, mu_r[v], 1);
                fb[v] = lane >= 1 ? s * (mu_r[v] - mu_l[v]) : 0.0;
            }
            double f[4], wlb[4], wrb[4], gface = 0.0;
            mc::hllc_vjp2(K, axis, left, rl, fb, f, wlb, wrb, &gface);
            // faces 0 .. extent-1 of this line belong to this tile
            const bool own_face = r >= 0 && r < (axis == 0 ? vw : vh);
            if (own_face) {
                gam += gface;
            }
            // Per variable: the cotangents of this cell's face values (RL from
            // its own, left face; RR from the next face, lane + 1), the WENO
            // VJP onto the stencil, and the gather of the stencil
            // contributions of cells c-2 .. c+2 into cell c.
            const int c = r;  // tile cell of this lane
            const bool own_cell = c >= 0 && c < (axis == 0 ? vw : vh);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const double rlb = lane >= 1 ? wrb[v] : 0.0;
                const double nx_l = __shfl_down_sync(0xffffffffu, wlb[v], 1);
                const double rrb = lane <= 30 ? nx_l : 0.0;
                // divergence of the flux, for the dt sensitivity
                const double fn = __shfl_down_sync(0xffffffffu, f[v], 1);
                if (own_cell) {
                    gdt += mu_r[v] * (f[v] - fn);
                }
                double st[5], sb[5];
#pragma unroll
                for (int o = 0; o < 5; ++o) {
                    st[o] = wat(v, o - 2);
                    sb[o] = 0.0;
                }
                mc::weno5z_vjp(st, rlb, rrb, sb);
                const double g = __shfl_down_sync(0xffffffffu, sb[0], 2) + __shfl_down_sync(0xffffffffu, sb[1], 1) +
                                 sb[2] + __shfl_up_sync(0xffffffffu, sb[3], 1) + __shfl_up_sync(0xffffffffu, sb[4], 2);
                if (own_cell) {
                    double* dst = axis == 0 ? &WB[(v * AT + line) * kBP + c] : &WB[(v * AT + c) * kBP + line];
                    *dst += g;
                }
            }
        }
        __syncthreads();
    }

    // primitive cotangents -> conserved cotangents; write lam, acc
    for (int it = threadIdx.x; it < AT * AT; it += kAThreads) {
        const int ty = it / AT, tx = it - ty * AT;
        if (tx >= vw || ty >= vh) {
            continue;
        }
        const int i = p.ng + x0 + tx, j = p.ng + y0 + ty;
        double q[4], wb[4], qb[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            q[v] = p.q[pidx(p, v, j, i)];
            wb[v] = WB[(v * AT + ty) * kBP + tx];
        }
        mc::prim_from_cons_vjp2(gamma, q, wb, qb, &gam);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const long long id = pidx(p, v, j, i);
            const double m = p.mu[id];
            double l = p.b * m + qb[v];
            if (p.add) {
                l += p.add[id];
            }
            p.lam[id] = l;
            if (p.acc_out) {
                p.acc_out[id] = (p.acc_in ? p.acc_in[id] : 0.0) + p.a * m;
            }
        }
    }
    const double sg = block_sum(gdt, red);
    const double sm = block_sum(gam, red);
    if (threadIdx.x == 0) {
        const int bid = blockIdx.y * gridDim.x + blockIdx.x;
        p.part_gdt[bid] = sg;
        p.part_gam[bid] = sm;
    }
}

// Fixed-order reduction of the per-CTA partial sums of one stage:
// step_gdt += (b / dx) * sum(part_gdt), gamma_bar += sum(part_gam).
__global__ void reduce_stage_kernel(const double* part_gdt, const double* part_gam, int n, double b_over_dx,
                                    double* step_gdt, double* gamma_bar) {
    __shared__ double rg[kAWarps], rm[kAWarps];
    double g = 0.0, m = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        g += part_gdt[k];
        m += part_gam[k];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        g += __shfl_xor_sync(0xffffffffu, g, o);
        m += __shfl_xor_sync(0xffffffffu, m, o);
    }
    if ((threadIdx.x & 31) == 0) {
        rg[threadIdx.x >> 5] = g;
        rm[threadIdx.x >> 5] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double G = 0.0, M = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            G += rg[w];
            M += rm[w];
        }
        *step_gdt += b_over_dx * G;
        *gamma_bar += M;
    }
}

// The arg-min cell as a key ordered like global cell indices over y slabs:
// (rank << 32) | local index, or the largest key when this rank holds none.
__global__ void argmin_key_kernel(const int* idx, int rank, long long* key) {
    *key = *idx == 0x7fffffff ? 0x7fffffffffffffffLL : ((long long)rank << 32) | (long long)*idx;
}

// Close one step of the reverse sweep: route the step's dt sensitivity to
// the arg-min cell (unless the output clamp fixed dt) on the rank that owns
// it, then clear it.
__global__ void dt_vjp_kernel(const double* q, int nx, int ng, int xc, int yc, double gamma, double dx,
                              double max_cfl, const long long* key, int rank, const int* clamped, double* step_gdt,
                              double* lam, double* gamma_bar) {
    const double g = *step_gdt;
    *step_gdt = 0.0;
    const long long k_ = *key;
    if (*clamped || k_ == 0x7fffffffffffffffLL || (int)(k_ >> 32) != rank || g == 0.0) {
        return;
    }
    const int c = (int)(k_ & 0xffffffffLL);
    const int xi = c % nx, yi = c / nx;
    const long long plane = (long long)xc * yc;
    const long long cell = (long long)(yi + ng) * xc + xi + ng;
    double qq[4], qb[4], gb = 0.0;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        qq[v] = q[v * plane + cell];
    }
    mc::cfl_dt_grad2(gamma, dx, qq, qb, &gb);
    const double k = g * max_cfl;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        lam[v * plane + cell] += k * qb[v];
    }
    *gamma_bar += k * gb;
}


__global__ void reciprocal_kernel(const double* x, double* out, long long n) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        out[k] = mc::arcp(x[k]);
    }
}

// Rows of the 4 variables between the padded state and contiguous
// [4][rows][xc] blocks, two blocks per launch: dst_b[v * dst_stride + k] =
// src_b[v * src_stride + k] for k < len, b = 0, 1.
__global__ void copy_rows_kernel(const double* src0, const double* src1, double* dst0, double* dst1,
                                 long long src_stride, long long dst_stride, long long len) {
    const long long n = 8 * len;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / (4 * len));
        const long long r = t - b * 4 * len;
        const int v = (int)(r / len);
        const long long k = r - v * len;
        (b ? dst1 : dst0)[v * dst_stride + k] = (b ? src1 : src0)[v * src_stride + k];
    }
}

__global__ void zero_kernel(double* p, long long n) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        p[k] = 0.0;
    }
}

} // namespace

struct mc_adjoint {
    mc_grid grid{};
    mc_scheme scheme{};
    int k = 20;                 // checkpoint interval
    int nx = 0, ny = 0;
    long long plane = 0;
    size_t state = 0;           // doubles per state
    double* ckpt = nullptr;     // checkpoints (grown on demand)
    int64_t ckpt_cap = 0;
    double* seg = nullptr;      // (3 k_eff + 1) states of the segment being reversed
    int64_t seg_cap = 0;        // segment length (steps) the buffer holds
    double* work_a = nullptr;   // forward stage buffers
    double* work_b = nullptr;
    double* lam[3] = {nullptr, nullptr, nullptr};
    double* acc = nullptr;
    double* dts = nullptr;
    double* mins = nullptr;
    int* clamped = nullptr;
    int64_t rec_cap = 0;
    int64_t n_steps = 0;        // steps of the recorded forward run
    DeviceBlock* blk = nullptr;
    DeviceBlock* blk_rec = nullptr;  // control block of the recompute (never done)
    double* part = nullptr;     // 2 x tiles partial sums
    double* scal = nullptr;     // [0] step g_dt, [1] gamma bar
    int* argmin = nullptr;
    long long* key = nullptr;   // arg-min key (argmin_key_kernel)
    int tiles = 0;
    bool recorded = false;
    // slab decomposition along y (mc_adjoint_set_slab_*)
    bool sliced = false;
    int rank = 0, world = 1;
    mc::SlabExchange* slab = nullptr;  // NCCL, or
    mc_comm_fn comm_fn = nullptr;      // the caller's hook
    void* comm_user = nullptr;
    long long halo_cap = 0;            // doubles per send / receive block: 4 (kAH + kMH) xc
    double* send = nullptr;            // [2][halo_cap]: to the rank below, to the rank above
    double* recv = nullptr;            // [2][halo_cap]: from the rank below, from the rank above
};

namespace {

mc_status afail(mc_status s, const std::string& msg) {
    mc::set_last_error(msg.c_str());
    return s;
}

#define MCA_CUDA(call, where)                                                              \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            return afail(MC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e_)); \
        }                                                                                  \
    } while (0)

StageParams fwd_params(const mc_adjoint* a) {
    StageParams p;
    std::memset(&p, 0, sizeof(p));
    p.xc = a->grid.xc;
    p.yc = a->grid.yc;
    p.zc = 1;
    p.ng = a->grid.ng;
    p.nx = a->nx;
    p.ny = a->ny;
    p.nz = 1;
    p.nvar = 4;
    p.plane = a->plane;
    p.dx = a->grid.dx;
    p.gamma = a->scheme.gamma;
    p.blk = a->blk;
    for (int f = 0; f < 6; ++f) {
        p.bc.kind[f] = f < 4 ? MC_BC_PERIODIC : MC_BC_USERFN;
    }
    if (a->sliced) {
        // the exchange fills the ghost rows between slabs
        p.bc.kind[2] = p.bc.kind[3] = MC_BC_USERFN;
    }
    return p;
}

mc_status comm_halo(mc_adjoint* a, long long count, cudaStream_t s) {
    double* slo = a->send;
    double* shi = a->send + a->halo_cap;
    double* rlo = a->recv;
    double* rhi = a->recv + a->halo_cap;
    if (a->slab) {
        const char* why = "";
        if (mc::slab_halo(a->slab, slo, shi, rlo, rhi, (size_t)count, s, &why) != cudaSuccess) {
            return afail(MC_ERR_CUDA, std::string("slab halo exchange: ") + why);
        }
        return MC_OK;
    }
    void* bufs[4] = {slo, shi, rlo, rhi};
    if (a->comm_fn(a->comm_user, MC_COMM_HALO, bufs, count, (void*)s) != 0) {
        return afail(MC_ERR_CUDA, "slab hook: halo exchange failed");
    }
    return MC_OK;
}

mc_status comm_reduce(mc_adjoint* a, mc_comm_op op, void* buf, cudaStream_t s) {
    if (a->slab) {
        const mc::SlabReduce r = op == MC_COMM_MIN_U64   ? mc::SlabReduce::kMinU64
                                 : op == MC_COMM_SUM_F64 ? mc::SlabReduce::kSumF64
                                                         : mc::SlabReduce::kMinI64;
        const char* why = "";
        if (mc::slab_all_reduce(a->slab, buf, 1, r, s, &why) != cudaSuccess) {
            return afail(MC_ERR_CUDA, std::string("slab all-reduce: ") + why);
        }
        return MC_OK;
    }
    void* bufs[4] = {buf, nullptr, nullptr, nullptr};
    if (a->comm_fn(a->comm_user, op, bufs, 1, (void*)s) != 0) {
        return afail(MC_ERR_CUDA, "slab hook: all-reduce failed");
    }
    return MC_OK;
}

int copy_blocks(long long len) {
    const long long b = (8 * len + 255) / 256;
    return (int)(b < 148 * 4 ? b : 148 * 4);
}

// Ghost rows between slabs: this slab's first / last ng rows to the ranks
// below / above, their bordering rows into its ghost rows.
mc_status exchange_ghosts(mc_adjoint* a, double* q, cudaStream_t s) {
    if (!a->sliced) {
        return MC_OK;
    }
    const long long xc = a->grid.xc, ng = a->grid.ng, ny = a->ny;
    const long long len = ng * xc;
    copy_rows_kernel<<<copy_blocks(len), 256, 0, s>>>(q + ng * xc, q + ny * xc, a->send, a->send + a->halo_cap,
                                                      a->plane, len, len);
    MCA_CUDA(cudaGetLastError(), "pack ghost rows");
    if (mc_status st = comm_halo(a, 4 * len, s)) {
        return st;
    }
    copy_rows_kernel<<<copy_blocks(len), 256, 0, s>>>(a->recv, a->recv + a->halo_cap, q, q + (ny + ng) * xc, len,
                                                      a->plane, len);
    MCA_CUDA(cudaGetLastError(), "unpack ghost rows");
    return MC_OK;
}

// The rows a stage's product reads beyond the slab: kAH rows of the stage
// input and kMH rows of its cotangent from each neighbour, into the receive
// blocks ([4][kAH][xc] then [4][kMH][xc] in each).
mc_status exchange_vjp_halo(mc_adjoint* a, const double* q, const double* mu, cudaStream_t s) {
    const long long xc = a->grid.xc, ng = a->grid.ng, ny = a->ny;
    const long long lq = kAH * xc, lm = kMH * xc;
    copy_rows_kernel<<<copy_blocks(lq), 256, 0, s>>>(q + ng * xc, q + (ng + ny - kAH) * xc, a->send,
                                                     a->send + a->halo_cap, a->plane, lq, lq);
    MCA_CUDA(cudaGetLastError(), "pack halo rows");
    copy_rows_kernel<<<copy_blocks(lm), 256, 0, s>>>(mu + ng * xc, mu + (ng + ny - kMH) * xc, a->send + 4 * lq,
                                                     a->send + a->halo_cap + 4 * lq, a->plane, lm, lm);
    MCA_CUDA(cudaGetLastError(), "pack cotangent halo rows");
    return comm_halo(a, a->halo_cap, s);
}

// The CFL minimum word of the forward's control block, reduced over the slabs.
mc_status reduce_cfl_word(mc_adjoint* a, cudaStream_t s) {
    if (!a->sliced) {
        return MC_OK;
    }
    return comm_reduce(a, MC_COMM_MIN_U64, &a->blk->cfl_min_bits, s);
}

// One SSPRK3 stage of the forward scheme (the fused FP64 kernel), then the
// ghost rows between slabs. The recompute of the reverse sweep runs on its
// own control block, which never marks the loop done.
mc_status fwd_stage(mc_adjoint* a, const double* in, const double* old_, double* out, int combo, int last,
                    const double* dt_dev, cudaStream_t s, bool recompute = false) {
    StageParams p = fwd_params(a);
    if (recompute) {
        p.blk = a->blk_rec;
    }
    p.q_in = in;
    p.q_old = old_;
    p.q_out = out;
    p.dt_dev = dt_dev;
    p.combo = combo;
    p.last = last;
    MCA_CUDA(mc::launch_stage_d2_fp64(p, MC_RECON_WENO5Z, MC_LIMITER_MONOTONIZED_CENTRAL, MC_RIEMANN_HLLC, 0, s),
             "forward stage");
    return exchange_ghosts(a, out, s);
}

mc_status grow(mc_adjoint* a, int64_t steps) {
    // the segment buffer: (3 k + 1) states for segments of k = min(interval, steps) steps
    const int64_t k_eff = steps < a->k ? (steps > 0 ? steps : 1) : a->k;
    if (k_eff > a->seg_cap) {
        cudaFree(a->seg);
        a->seg = nullptr;
        a->seg_cap = 0;
        MCA_CUDA(cudaMalloc(&a->seg, sizeof(double) * a->state * (3 * (size_t)k_eff + 1)), "alloc segment");
        a->seg_cap = k_eff;
    }
    // the records hold steps + 1 entries (a run of 0 steps still records its first dt)
    if (a->dts && a->mins && a->clamped && a->ckpt && steps <= a->rec_cap) {
        return MC_OK;
    }
    cudaFree(a->dts);
    cudaFree(a->mins);
    cudaFree(a->clamped);
    cudaFree(a->ckpt);
    a->dts = a->mins = a->ckpt = nullptr;
    a->clamped = nullptr;
    const int64_t nck = steps / a->k + 1;
    MCA_CUDA(cudaMalloc(&a->dts, sizeof(double) * (steps + 1)), "alloc");
    MCA_CUDA(cudaMalloc(&a->mins, sizeof(double) * (steps + 1)), "alloc");
    MCA_CUDA(cudaMalloc(&a->clamped, sizeof(int) * (steps + 1)), "alloc");
    MCA_CUDA(cudaMalloc(&a->ckpt, sizeof(double) * a->state * nck), "alloc checkpoints");
    a->rec_cap = steps;
    return MC_OK;
}

mc_status vjp_stage(mc_adjoint* a, const double* q, const double* mu, double* lam, const double* add,
                    const double* acc_in, double* acc_out, double coef_a, double coef_b, const double* dt,
                    cudaStream_t s) {
    VjpParams p;
    std::memset(&p, 0, sizeof(p));
    p.q = q;
    p.mu = mu;
    p.lam = lam;
    p.add = add;
    p.acc_in = acc_in;
    p.acc_out = acc_out;
    p.dt = dt;
    if (a->sliced) {
        if (mc_status st = exchange_vjp_halo(a, q, mu, s)) {
            return st;
        }
        p.qlo = a->recv;
        p.mlo = a->recv + 4 * kAH * (long long)a->grid.xc;
        p.qhi = a->recv + a->halo_cap;
        p.mhi = p.qhi + 4 * kAH * (long long)a->grid.xc;
    }
    p.a = coef_a;
    p.b = coef_b;
    p.dx = a->grid.dx;
    p.gamma = a->scheme.gamma;
    p.nx = a->nx;
    p.ny = a->ny;
    p.ng = a->grid.ng;
    p.xc = a->grid.xc;
    p.yc = a->grid.yc;
    p.part_gdt = a->part;
    p.part_gam = a->part + a->tiles;
    const dim3 grid((a->nx + kTile - 1) / kTile, (a->ny + kTile - 1) / kTile);
    stage_vjp_kernel<kTile><<<grid, kAThreads, VjpTile<kTile>::smem_bytes(), s>>>(p);
    MCA_CUDA(cudaGetLastError(), "stage vjp");
    reduce_stage_kernel<<<1, 256, 0, s>>>(a->part, a->part + a->tiles, a->tiles, coef_b / a->grid.dx, a->scal,
                                          a->scal + 1);
    MCA_CUDA(cudaGetLastError(), "reduce");
    return MC_OK;
}

// Checks and buffers shared by both forms of the slab decomposition.
mc_status slab_prepare(mc_adjoint* a, int32_t rank, int32_t world) {
    if (!a || world < 1 || rank < 0 || rank >= world) {
        return afail(MC_ERR_INVALID_ARGUMENT, "null adjoint or rank outside [0, world)");
    }
    if (a->sliced) {
        return afail(MC_ERR_INVALID_ARGUMENT, "the adjoint already holds a slab decomposition");
    }
    if (a->recorded) {
        return afail(MC_ERR_INVALID_ARGUMENT, "join the slab decomposition before the forward run");
    }
    if (a->ny < kAH || a->ny < a->grid.ng) {
        return afail(MC_ERR_INVALID_ARGUMENT, "a slab needs at least max(5, ng) rows");
    }
    // one block holds the VJP halos ([4][kAH][xc] + [4][kMH][xc]) or ng ghost rows
    a->halo_cap = 4LL * (kAH + kMH > a->grid.ng ? kAH + kMH : a->grid.ng) * a->grid.xc;
    if (!a->send) {
        MCA_CUDA(cudaMalloc(&a->send, sizeof(double) * 2 * (size_t)a->halo_cap), "alloc halo");
    }
    if (!a->recv) {
        MCA_CUDA(cudaMalloc(&a->recv, sizeof(double) * 2 * (size_t)a->halo_cap), "alloc halo");
    }
    return MC_OK;
}

} // namespace

extern "C" {

mc_status mc_adjoint_create(const mc_grid* grid, const mc_scheme* scheme, int32_t checkpoint_every,
                            mc_adjoint** out) {
    if (!grid || !scheme || !out || checkpoint_every < 1) {
        return afail(MC_ERR_INVALID_ARGUMENT, "null argument or checkpoint interval < 1");
    }
    *out = nullptr;
    const mc_grid& g = *grid;
    const mc_scheme& s = *scheme;
    if (g.num_dim != 2 || g.num_tracers != 0 || s.reconstruction != MC_RECON_WENO5Z ||
        s.riemann_solver != MC_RIEMANN_HLLC || s.time_stepper != MC_STEPPER_SSPRK3 ||
        s.precision != MC_PRECISION_FP64) {
        return afail(MC_ERR_UNSUPPORTED, "the adjoint covers 2D WENO5-Z + HLLC + SSPRK3 in FP64 without tracers");
    }
    for (int f = 0; f < 4; ++f) {
        if (g.bc[f] != MC_BC_PERIODIC) {
            return afail(MC_ERR_UNSUPPORTED, "the adjoint covers periodic faces");
        }
    }
    if (g.ng < 3 || g.zc != 1 || g.xc - 2 * g.ng < kAH || g.yc - 2 * g.ng < kAH || !(g.dx > 0.0)) {
        return afail(MC_ERR_INVALID_ARGUMENT, "bad extents (ng >= 3, at least 5 interior cells per axis)");
    }
    mc_adjoint* a = new (std::nothrow) mc_adjoint();
    if (!a) {
        return afail(MC_ERR_OUT_OF_MEMORY, "host allocation");
    }
    a->grid = g;
    a->scheme = s;
    a->k = checkpoint_every;
    a->nx = g.xc - 2 * g.ng;
    a->ny = g.yc - 2 * g.ng;
    a->plane = (long long)g.xc * g.yc;
    a->state = 4 * (size_t)a->plane;
    a->tiles = ((a->nx + kTile - 1) / kTile) * ((a->ny + kTile - 1) / kTile);
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) {
            e = cudaMalloc(p, bytes);
        }
    };
    const size_t sb = sizeof(double) * a->state;
    alloc((void**)&a->work_a, sb);
    alloc((void**)&a->work_b, sb);
    for (auto& l : a->lam) {
        alloc((void**)&l, sb);
    }
    alloc((void**)&a->acc, sb);
    alloc((void**)&a->blk, sizeof(DeviceBlock));
    alloc((void**)&a->blk_rec, sizeof(DeviceBlock));
    if (e == cudaSuccess) {
        e = cudaMemset(a->blk_rec, 0, sizeof(DeviceBlock));
    }
    alloc((void**)&a->part, sizeof(double) * 2 * a->tiles);
    alloc((void**)&a->scal, sizeof(double) * 2);
    alloc((void**)&a->argmin, sizeof(int));
    alloc((void**)&a->key, sizeof(long long));
    if (e == cudaSuccess) {
        e = cudaFuncSetAttribute(stage_vjp_kernel<kTile>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)VjpTile<kTile>::smem_bytes());
    }
    if (e != cudaSuccess) {
        mc_adjoint_destroy(a);
        return afail(e == cudaErrorMemoryAllocation ? MC_ERR_OUT_OF_MEMORY : MC_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = a;
    return MC_OK;
}

mc_status mc_adjoint_destroy(mc_adjoint* a) {
    if (!a) {
        return MC_OK;
    }
    cudaFree(a->ckpt);
    cudaFree(a->seg);
    cudaFree(a->work_a);
    cudaFree(a->work_b);
    for (auto l : a->lam) {
        cudaFree(l);
    }
    cudaFree(a->acc);
    cudaFree(a->dts);
    cudaFree(a->mins);
    cudaFree(a->clamped);
    cudaFree(a->blk);
    cudaFree(a->blk_rec);
    cudaFree(a->part);
    cudaFree(a->scal);
    cudaFree(a->argmin);
    cudaFree(a->key);
    cudaFree(a->send);
    cudaFree(a->recv);
    mc::slab_destroy(a->slab);
    delete a;
    return MC_OK;
}

mc_status mc_adjoint_forward(mc_adjoint* a, double* Q, const mc_clock* clock, int64_t n_steps, void* stream) {
    if (!a || !Q || !clock || n_steps < 0) {
        return afail(MC_ERR_INVALID_ARGUMENT, "null argument or negative step count");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    if (mc_status st = grow(a, n_steps)) {
        return st;
    }
    const size_t sb = sizeof(double) * a->state;
    MCA_CUDA(mc::launch_clock_init(a->blk, clock->time, clock->max_time, clock->prev_output_time,
                                   clock->output_delta, a->scheme.max_cfl, s),
             "clock init");
    if (mc_status st = exchange_ghosts(a, Q, s)) {
        return st;
    }
    StageParams p = fwd_params(a);
    p.q_in = Q;
    MCA_CUDA(mc::launch_cfl_min(p, 2, s), "cfl");
    if (mc_status st = reduce_cfl_word(a, s)) {
        return st;
    }
    MCA_CUDA(mc::launch_record_clock(a->blk, 1, a->dts, a->mins, a->clamped, 0, s), "clock");
    for (int64_t n = 0; n < n_steps; ++n) {
        if (n % a->k == 0) {
            MCA_CUDA(cudaMemcpyAsync(a->ckpt + (n / a->k) * a->state, Q, sb, cudaMemcpyDeviceToDevice, s), "checkpoint");
        }
        const double* dt = a->dts + n;
        if (mc_status st = fwd_stage(a, Q, Q, a->work_a, mc::kAdd, 0, dt, s)) {
            return st;
        }
        if (mc_status st = fwd_stage(a, a->work_a, Q, a->work_b, mc::kSsp3Second, 0, dt, s)) {
            return st;
        }
        if (mc_status st = fwd_stage(a, a->work_b, Q, Q, mc::kSsp3Final, 1, dt, s)) {
            return st;
        }
        if (mc_status st = reduce_cfl_word(a, s)) {
            return st;
        }
        MCA_CUDA(mc::launch_record_clock(a->blk, 0, a->dts, a->mins, a->clamped, n + 1, s), "clock");
        MCA_CUDA(cudaGetLastError(), "clock");
    }
    a->n_steps = n_steps;
    a->recorded = true;
    return MC_OK;
}

mc_status mc_adjoint_backward(mc_adjoint* a, double* lambda, double* dgamma, void* stream) {
    if (!a || !lambda) {
        return afail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    if (!a->recorded) {
        return afail(MC_ERR_INVALID_ARGUMENT, "no recorded forward run");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    const size_t sb = sizeof(double) * a->state;
    zero_kernel<<<64, 256, 0, s>>>(a->scal, 2);
    MCA_CUDA(cudaMemcpyAsync(a->lam[0], lambda, sb, cudaMemcpyDeviceToDevice, s), "lambda in");
    double* L3 = a->lam[0];
    double* L2 = a->lam[1];
    double* L1 = a->lam[2];
    const int64_t nseg = (a->n_steps + a->k - 1) / a->k;
    for (int64_t sg = nseg - 1; sg >= 0; --sg) {
        const int64_t n0 = sg * a->k;
        const int64_t len = (a->n_steps - n0) < a->k ? (a->n_steps - n0) : a->k;
        // recompute the segment's stage states from its checkpoint
        MCA_CUDA(cudaMemcpyAsync(a->seg, a->ckpt + sg * a->state, sb, cudaMemcpyDeviceToDevice, s), "checkpoint");
        for (int64_t j = 0; j < len; ++j) {
            double* q0 = a->seg + (3 * j) * a->state;
            double* q1 = q0 + a->state;
            double* q2 = q1 + a->state;
            double* q3 = q2 + a->state;
            const double* dt = a->dts + n0 + j;
            if (mc_status st = fwd_stage(a, q0, q0, q1, mc::kAdd, 0, dt, s, true)) {
                return st;
            }
            if (mc_status st = fwd_stage(a, q1, q0, q2, mc::kSsp3Second, 0, dt, s, true)) {
                return st;
            }
            if (mc_status st = fwd_stage(a, q2, q0, q3, mc::kSsp3Final, 0, dt, s, true)) {
                return st;
            }
        }
        // reverse the segment's steps
        for (int64_t j = len - 1; j >= 0; --j) {
            const double* q0 = a->seg + (3 * j) * a->state;
            const double* q1 = q0 + a->state;
            const double* q2 = q1 + a->state;
            const double* dt = a->dts + n0 + j;
            // Q3 = 1/3 Q0 + 2/3 (Q2 + dt L(Q2))
            if (mc_status st = vjp_stage(a, q2, L3, L2, nullptr, nullptr, a->acc, 1.0 / 3.0, 2.0 / 3.0, dt, s)) {
                return st;
            }
            // Q2 = 3/4 Q0 + 1/4 (Q1 + dt L(Q1))
            if (mc_status st = vjp_stage(a, q1, L2, L1, nullptr, a->acc, a->acc, 0.75, 0.25, dt, s)) {
                return st;
            }
            // Q1 = Q0 + dt L(Q0); lam0 gathers the Q0 terms of all stages
            if (mc_status st = vjp_stage(a, q0, L1, L3, a->acc, nullptr, nullptr, 0.0, 1.0, dt, s)) {
                return st;
            }
            // dt of this step = max_cfl * CFL minimum of Q0
            MCA_CUDA(mc::launch_cfl_argmin(q0, a->nx, a->ny, a->grid.ng, a->grid.xc, a->grid.yc, a->scheme.gamma,
                                           a->grid.dx, a->mins + n0 + j, a->argmin, s),
                     "arg-min");
            argmin_key_kernel<<<1, 1, 0, s>>>(a->argmin, a->rank, a->key);
            if (a->sliced) {
                // the lowest global arg-min cell and the step's whole dt sensitivity
                if (mc_status st = comm_reduce(a, MC_COMM_MIN_I64, a->key, s)) {
                    return st;
                }
                if (mc_status st = comm_reduce(a, MC_COMM_SUM_F64, a->scal, s)) {
                    return st;
                }
            }
            dt_vjp_kernel<<<1, 1, 0, s>>>(q0, a->nx, a->grid.ng, a->grid.xc, a->grid.yc, a->scheme.gamma,
                                          a->grid.dx, a->scheme.max_cfl, a->key, a->rank, a->clamped + n0 + j,
                                          a->scal, L3, a->scal + 1);
            MCA_CUDA(cudaGetLastError(), "dt vjp");
        }
    }
    if (a->sliced) {
        if (mc_status st = comm_reduce(a, MC_COMM_SUM_F64, a->scal + 1, s)) {
            return st;
        }
    }
    MCA_CUDA(cudaMemcpyAsync(lambda, L3, sb, cudaMemcpyDeviceToDevice, s), "lambda out");
    if (dgamma) {
        MCA_CUDA(cudaMemcpyAsync(dgamma, a->scal + 1, sizeof(double), cudaMemcpyDeviceToHost, s), "dgamma");
        MCA_CUDA(cudaStreamSynchronize(s), "sync");
    }
    return MC_OK;
}

mc_status mc_adjoint_set_slab_decomposition(mc_adjoint* a, const uint8_t* id, int32_t rank, int32_t world) {
    if (!id) {
        return afail(MC_ERR_INVALID_ARGUMENT, "null id");
    }
    if (mc_status st = slab_prepare(a, rank, world)) {
        return st;
    }
    const char* why = "";
    mc::SlabExchange* x = mc::slab_create(id, rank, world, 1, a->ny, a->grid.ng, a->grid.xc, a->grid.yc, 1, 4,
                                          true, &why);
    if (!x) {
        return afail(MC_ERR_CUDA, std::string("slab communicator: ") + why);
    }
    a->slab = x;
    a->rank = rank;
    a->world = world;
    a->sliced = true;
    return MC_OK;
}

mc_status mc_adjoint_set_slab_hook(mc_adjoint* a, mc_comm_fn fn, void* user, int32_t rank, int32_t world) {
    if (!fn) {
        return afail(MC_ERR_INVALID_ARGUMENT, "null hook");
    }
    if (mc_status st = slab_prepare(a, rank, world)) {
        return st;
    }
    a->comm_fn = fn;
    a->comm_user = user;
    a->rank = rank;
    a->world = world;
    a->sliced = true;
    return MC_OK;
}

mc_status mc_debug_reverse_reciprocal(const double* x, double* out, int64_t n, void* stream) {
    if (!x || !out || n < 0) {
        return afail(MC_ERR_INVALID_ARGUMENT, "null argument or negative count");
    }
    if (n > 0) {
        reciprocal_kernel<<<148 * 4, 256, 0, (cudaStream_t)stream>>>(x, out, n);
        MCA_CUDA(cudaGetLastError(), "reciprocal");
    }
    return MC_OK;
}

} // extern "C"
