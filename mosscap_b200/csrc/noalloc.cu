// mc_time_step_noalloc: one SSPRK step that allocates no device memory.
//
// mc_create allocates two state-sized stage buffers (and, in 3D, a buffer
// for the x+y divergence) with cudaMalloc. Some callers cannot do that:
// a code whose device memory is owned by a pool allocator sized at start-up
// (Mosscap itself runs on a YAKL/Kokkos pool), or one that must not call
// cudaMalloc/cudaFree in the middle of a run because those calls synchronise
// the device. For them this entry point takes the stage buffers from one
// file-scope __device__ array of fixed size instead, so it never allocates.
//
// The array is kNoAllocScratchBytes (16 MiB) and lives for the whole process
// on every GPU that loads the library. Problems whose stage buffers do not
// fit are rejected with MC_ERR_OUT_OF_MEMORY. All calls share the array:
// two calls whose work overlaps on the GPU (different streams, or different
// host threads on one device) race on it and must not be issued.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "launch.h"
#include "mosscap_b200.h"

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;
constexpr size_t kNoAllocScratchDoubles = kNoAllocScratchBytes / sizeof(double);
constexpr int kMaxDevices = 64;

// The shared scratch: stage buffers A and B, then (3D) the x+y divergence.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
// The control block the stage kernels reduce into (CFL minimum, flags).
static __device__ __align__(256) mc::DeviceBlock g_noalloc_block;

// Device addresses of the two arrays, looked up once per device. In host
// code g_noalloc_scratch names a host-side stand-in, never the device memory.
struct DeviceSymbols {
    double* scratch = nullptr;
    mc::DeviceBlock* block = nullptr;
    bool ready = false;
};
DeviceSymbols g_symbols[kMaxDevices];
std::mutex g_symbols_mutex;

mc_status fail(mc_status s, const char* msg) {
    mc::set_last_error(msg);
    return s;
}

mc_status fail_cuda(cudaError_t e, const char* where) {
    char msg[256];
    std::snprintf(msg, sizeof(msg), "%s: %s", where, cudaGetErrorString(e));
    mc::set_last_error(msg);
    return MC_ERR_CUDA;
}

// First call on a device: resolve the device addresses of the static arrays
// with that device current and check the return codes.
mc_status device_symbols(DeviceSymbols** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        return fail_cuda(e, "cudaGetDevice");
    }
    if (dev < 0 || dev >= kMaxDevices) {
        return fail(MC_ERR_UNSUPPORTED, "device ordinal above 63");
    }
    std::lock_guard<std::mutex> lock(g_symbols_mutex);
    DeviceSymbols& s = g_symbols[dev];
    if (!s.ready) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            return fail_cuda(e, "cudaGetSymbolAddress(scratch)");
        }
        s.scratch = static_cast<double*>(p);
        e = cudaGetSymbolAddress(&p, g_noalloc_block);
        if (e != cudaSuccess) {
            return fail_cuda(e, "cudaGetSymbolAddress(block)");
        }
        s.block = static_cast<mc::DeviceBlock*>(p);
        s.ready = true;
    }
    *out = &s;
    return MC_OK;
}

int halo_of_recon(int rec) {
    return rec == MC_RECON_FOG ? 1 : rec == MC_RECON_MUSCL ? 2 : 3;
}

mc_status validate(const mc_grid& g, const mc_scheme& s) {
    if (g.num_dim < 1 || g.num_dim > 3) {
        return fail(MC_ERR_INVALID_ARGUMENT, "num_dim must be 1, 2 or 3");
    }
    if (s.reconstruction < 0 || s.reconstruction > 3 || s.slope_limiter < 0 || s.slope_limiter > 2 ||
        s.riemann_solver < 0 || s.riemann_solver > 2 || s.time_stepper < 0 || s.time_stepper > 2 ||
        s.precision < 0 || s.precision > 1) {
        return fail(MC_ERR_INVALID_ARGUMENT, "scheme enum out of range");
    }
    if (g.ng < halo_of_recon(s.reconstruction) || g.ng > mc::kMaxGhost) {
        return fail(MC_ERR_INVALID_ARGUMENT, "ng below the reconstruction's need or above 8");
    }
    const int ext[3] = {g.xc, g.yc, g.zc};
    for (int a = 0; a < 3; ++a) {
        if (a < g.num_dim ? (ext[a] - 2 * g.ng < g.ng) : (ext[a] != 1)) {
            return fail(MC_ERR_INVALID_ARGUMENT, "bad extents: each active axis needs ng interior cells");
        }
    }
    if (g.num_tracers < 0 || 2 + g.num_dim + g.num_tracers > mc::kMaxVars) {
        return fail(MC_ERR_INVALID_ARGUMENT, "too many variables (at most 8)");
    }
    if (!(g.dx > 0.0) || !std::isfinite(g.dx) || !std::isfinite(s.gamma)) {
        return fail(MC_ERR_INVALID_ARGUMENT, "dx and gamma must be finite (dx > 0)");
    }
    for (int f = 0; f < 2 * g.num_dim; ++f) {
        // no context, hence no user boundary hook: every face must be built in
        if (g.bc[f] < 0 || g.bc[f] >= MC_BC_USERFN) {
            return fail(MC_ERR_INVALID_ARGUMENT, "boundary kind must be a built-in one");
        }
        if (g.bc[f] == MC_BC_CONSTANT && 2 + g.num_dim + g.num_tracers > 5) {
            return fail(MC_ERR_UNSUPPORTED, "constant boundaries hold at most 5 variables");
        }
    }
    for (int a = 0; a < g.num_dim; ++a) {
        if ((g.bc[2 * a] == MC_BC_PERIODIC) != (g.bc[2 * a + 1] == MC_BC_PERIODIC)) {
            return fail(MC_ERR_INVALID_ARGUMENT, "periodic boundaries come in pairs");
        }
    }
    return MC_OK;
}

cudaError_t launch(const mc_grid& g, const mc_scheme& s, const mc::StageParams& p, int pass, cudaStream_t st) {
    const bool f32 = s.precision == MC_PRECISION_FP32_COMPENSATED;
    const int r = s.reconstruction, l = s.slope_limiter, rs = s.riemann_solver;
    if (g.num_dim == 1) {
        return f32 ? mc::launch_stage_d1_fp32(p, r, l, rs, pass, st) : mc::launch_stage_d1_fp64(p, r, l, rs, pass, st);
    }
    if (g.num_dim == 2) {
        return f32 ? mc::launch_stage_d2_fp32(p, r, l, rs, pass, st) : mc::launch_stage_d2_fp64(p, r, l, rs, pass, st);
    }
    return f32 ? mc::launch_stage_d3_fp32(p, r, l, rs, pass, st) : mc::launch_stage_d3_fp64(p, r, l, rs, pass, st);
}

} // namespace

extern "C" {

mc_status mc_time_step_noalloc(const mc_grid* grid, const mc_scheme* scheme, double* Q, double dt, void* stream) {
    if (!grid || !scheme || !Q) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) {
        return fail(MC_ERR_INVALID_ARGUMENT, "dt must be positive and finite");
    }
    const mc_grid& g = *grid;
    const mc_scheme& s = *scheme;
    if (mc_status st = validate(g, s)) {
        return st;
    }
    const int nx = g.xc - 2 * g.ng;
    const int ny = g.num_dim > 1 ? g.yc - 2 * g.ng : 1;
    const int nz = g.num_dim > 2 ? g.zc - 2 * g.ng : 1;
    const int nvar = 2 + g.num_dim + g.num_tracers;
    const size_t state = size_t(nvar) * size_t(g.xc) * size_t(g.yc) * size_t(g.zc);
    const size_t div = g.num_dim == 3 ? size_t(nvar) * size_t(nx) * size_t(ny) * size_t(nz) : 0;
    if (2 * state + div > kNoAllocScratchDoubles) {
        return fail(MC_ERR_OUT_OF_MEMORY,
                    "mc_time_step_noalloc: the problem needs more than the 16 MiB static scratch "
                    "(two states, plus the x+y divergence in 3D)");
    }
    DeviceSymbols* sym = nullptr;
    if (mc_status st = device_symbols(&sym)) {
        return st;
    }
    double* bufs[3] = {Q, sym->scratch, sym->scratch + state};
    // the same stage plan as the context path (launch.h)
    const mc::StagePlan plan = mc::plan_for(s.time_stepper);
    const cudaStream_t cs = static_cast<cudaStream_t>(stream);
    for (int k = 0; k < plan.n; ++k) {
        mc::StageParams p;
        std::memset(&p, 0, sizeof(p));
        p.q_in = bufs[plan.in[k]];
        p.q_old = Q;
        p.q_out = bufs[plan.out[k]];
        p.dqxy = g.num_dim == 3 ? sym->scratch + 2 * state : nullptr;
        p.xc = g.xc;
        p.yc = g.yc;
        p.zc = g.zc;
        p.ng = g.ng;
        p.nx = nx;
        p.ny = ny;
        p.nz = nz;
        p.nvar = nvar;
        p.ntracer = g.num_tracers;
        p.plane = (long long)g.xc * g.yc * g.zc;
        p.dx = g.dx;
        p.gamma = s.gamma;
        p.dt = dt;
        p.dt_dev = nullptr;
        p.combo = plan.combo[k];
        p.last = k == plan.n - 1;
        // the block keeps the last call's contents: the first stage clears the
        // CFL-minimum cell that the last stage reduces into
        p.reset_min = k == 0;
        p.blk = sym->block;
        for (int f = 0; f < 6; ++f) {
            p.bc.kind[f] = f < 2 * g.num_dim ? g.bc[f] : MC_BC_USERFN;
            for (int v = 0; v < mc::kMaxVars; ++v) {
                p.bc.cval[f][v] = v < 5 ? g.bc_const[f][v] : 0.0;
            }
        }
        cudaError_t e = launch(g, s, p, 0, cs);
        if (e == cudaSuccess && g.num_dim == 3) {
            p.reset_min = 0;
            e = launch(g, s, p, 1, cs);
        }
        if (e != cudaSuccess) {
            return fail_cuda(e, "stage launch");
        }
    }
    return MC_OK;
}

} // extern "C"
