// Batches of independent problems (mc_batch_* in include/mosscap_b200.h):
// work lists, per-problem clocks, the captured CUDA graph of one step and
// the schedule autotuner. Compiled with -fmad=false (the CFL bound and the
// clock arithmetic are bit-identical to the single-problem path).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "batch_launch.h"
#include "launch.h"
#include "mosscap_b200.h"

using mc::BatchItem2d;
using mc::BatchStageParams;
using mc::BatchTask1d;
using mc::DeviceBlock;
using mc::StageParams;

struct mc_batch {
    int n = 0;
    mc_scheme scheme{};
    int64_t pool_doubles = 0;
    std::vector<mc_batch_problem> problems;
    std::vector<StageParams> params;     // host copy of the per-problem parameters
    std::vector<long long> cells;        // cells per problem (ghosts included) for ordering
    StageParams* d_params = nullptr;
    long long* d_offsets = nullptr;
    StageParams* d_stage = nullptr;      // per stage, every problem's parameters bound to a pool (bind_stages)
    const double* stage_pool = nullptr;  // the pool d_stage is bound to
    DeviceBlock* d_blocks = nullptr;
    BatchItem2d* d_items2d = nullptr;
    int n2d = 0;
    BatchTask1d* d_tasks1d = nullptr;
    int ntasks1d = 0;
    int tasks_segs = 0;                  // segments per task the 1D list was built with
    int* d_counters = nullptr;           // one work counter per stage and part (kCounters)
    int* d_finished = nullptr;           // per stage and problem: work items finished (ghost fill)
    int* d_items_of = nullptr;           // per problem: its work items in a stage
    std::vector<int> tiles_of;           // per problem: its 2D tiles (0 for 1D problems)
    double* buf_a = nullptr;
    double* buf_b = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    cudaGraphExec_t graph = nullptr;
    const double* graph_pool = nullptr;
    int graph_key[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bool clocks_ready = false;
    const double* clocks_pool = nullptr;
    // schedule: one launch per stage over both work lists (merged: grid_all,
    // dynamic_all), or the 2D-tile launch (grid, dynamic) and the 1D launch
    // (grid1d, dynamic1d); segs = 30-cell segments per warp task
    bool merged = true;
    int grid_all = 0;
    int dynamic_all = 1;
    int grid = 0;
    int dynamic = 1;
    int grid1d = 0;
    int dynamic1d = 1;
    int segs = 2;
    int sms = 148;
    int occupancy = 1;      // resident CTAs per SM of the 2D-tile kernel
    int occupancy1d = 1;    // of the 1D kernel
    int occupancy_all = 1;  // and of the merged kernel
};

namespace {

inline int cdiv(long long a, long long b) {
    return (int)((a + b - 1) / b);
}

constexpr int kCounters = 8;  // 4 stages x 2 parts

mc_status bfail(mc_status s, const std::string& msg) {
    mc::set_last_error(msg.c_str());
    return s;
}

mc_status bcuda(cudaError_t e, const char* where) {
    return bfail(MC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define MCB_CUDA(call, where)            \
    do {                                 \
        cudaError_t e_ = (call);         \
        if (e_ != cudaSuccess) {         \
            return bcuda(e_, where);     \
        }                                \
    } while (0)

// stage plans (source/TimeStepping.cpp): input / output pool per stage
// (0 = caller's pool, 1 = A, 2 = B) and the combination
struct Plan {
    int n;
    int in[4], out[4], combo[4];
};
Plan plan_for(int stepper) {
    switch (stepper) {
        case MC_STEPPER_RK2:
            return {2, {0, 1}, {1, 0}, {mc::kAdd, mc::kRk2Final}};
        case MC_STEPPER_SSPRK3:
            return {3, {0, 1, 2}, {1, 2, 0}, {mc::kAdd, mc::kSsp3Second, mc::kSsp3Final}};
        default:
            return {4, {0, 1, 2, 1}, {1, 2, 1, 0}, {mc::kHalfAdd, mc::kHalfAdd, mc::kSsp4Third, mc::kHalfAdd}};
    }
}

// CFL minimum over every cell (ghosts included) of every problem, one CTA
// per problem (source/Hydro.cpp:209-229).
template <int NDIM>
__device__ void cfl_cells(const StageParams& p, const double* q, double& m, unsigned& flags) {
    constexpr int nh = 2 + NDIM;
    for (long long c = threadIdx.x; c < p.plane; c += blockDim.x) {
        double qq[nh], w[nh];
        bool fin = true;
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            qq[v] = q[v * p.plane + c];
            fin = fin && isfinite(qq[v]);
        }
        mc::prim_from_cons<NDIM>(p.gamma, qq, w);
        flags |= mc::state_flags(w[0], w[nh - 1], fin);
        m = mc::smin(mc::cfl_dt<NDIM>(p.gamma, p.dx, w), m);
    }
}

__global__ void __launch_bounds__(256) batch_cfl_kernel(const StageParams* probs, const long long* offs,
                                                        const double* pool) {
    __shared__ double red_d[8];
    __shared__ unsigned red_u[8];
    const StageParams& p = probs[blockIdx.x];
    const double* q = pool + offs[blockIdx.x];
    double m = __longlong_as_double((long long)mc::kInfBits);
    unsigned flags = 0;
    if (p.yc == 1) {
        cfl_cells<1>(p, q, m, flags);
    } else {
        cfl_cells<2>(p, q, m, flags);
    }
    mc::block_publish(m, flags, true, p.blk, red_d, red_u);
}

// One thread per problem: close its step (unless first) and pick its next
// dt; outputs only advance the problem's clock. Thread 0 also resets the
// work counters of the next step's stage launches, and each thread its
// problem's finished-item counts.
__global__ void batch_clock_kernel(DeviceBlock* blocks, int n, int first, int* counters, int* finished) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        for (int c = 0; c < kCounters; ++c) {
            counters[c] = 0;
        }
    }
    if (i < n) {
        for (int st = 0; st < 4; ++st) {
            finished[st * n + i] = 0;
        }
        mc::advance_clock(&blocks[i], nullptr, first != 0, false);
    }
}

size_t state_doubles(const mc_grid& g) {
    return size_t(2 + g.num_dim) * size_t(g.xc) * size_t(g.yc);
}

mc_status validate_problem(const mc_batch_problem& pr, const mc_scheme& s, int64_t pool_doubles) {
    const mc_grid& g = pr.grid;
    if (g.num_dim != 1 && g.num_dim != 2) {
        return bfail(MC_ERR_UNSUPPORTED, "batch problems are 1D or 2D");
    }
    if (g.num_tracers != 0) {
        return bfail(MC_ERR_UNSUPPORTED, "batch problems carry no tracers");
    }
    const int need = s.reconstruction == MC_RECON_FOG ? 1 : s.reconstruction == MC_RECON_MUSCL ? 2 : 3;
    if (g.ng < need || g.ng > mc::kMaxGhost || g.zc != 1 || (g.num_dim == 1 && g.yc != 1)) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "bad ghost count or extents");
    }
    if (g.xc - 2 * g.ng < g.ng || (g.num_dim == 2 && g.yc - 2 * g.ng < g.ng)) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "each active axis needs at least ng interior cells");
    }
    for (int f = 0; f < 2 * g.num_dim; ++f) {
        if (g.bc[f] < 0 || g.bc[f] >= MC_BC_CONSTANT) {
            return bfail(MC_ERR_UNSUPPORTED, "batch problems use wall/periodic/symmetric/diode/zerograd faces");
        }
    }
    for (int a = 0; a < g.num_dim; ++a) {
        if ((g.bc[2 * a] == MC_BC_PERIODIC) != (g.bc[2 * a + 1] == MC_BC_PERIODIC)) {
            return bfail(MC_ERR_INVALID_ARGUMENT, "periodic boundaries come in pairs");
        }
    }
    if (!(g.dx > 0.0) || pr.offset < 0 || pr.offset + (int64_t)state_doubles(g) > pool_doubles) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "dx <= 0 or problem outside the pool");
    }
    return MC_OK;
}

cudaError_t launch_stage(const mc_batch* b, const BatchStageParams& bp, int part, int grid, cudaStream_t s,
                         int* occ) {
    const bool f32 = b->scheme.precision == MC_PRECISION_FP32_COMPENSATED;
    const int r = b->scheme.reconstruction, l = b->scheme.slope_limiter, rs = b->scheme.riemann_solver;
    return f32 ? mc::launch_batch_stage_fp32(bp, r, l, rs, part, grid, s, occ)
               : mc::launch_batch_stage_fp64(bp, r, l, rs, part, grid, s, occ);
}

// 1D task list: consecutive groups of `segs` 30-cell segments per problem,
// biggest problems first.
mc_status build_tasks(mc_batch* b, int segs) {
    if (b->tasks_segs == segs && b->d_tasks1d) {
        return MC_OK;
    }
    std::vector<int> order;
    for (int i = 0; i < b->n; ++i) {
        if (b->problems[i].grid.num_dim == 1) {
            order.push_back(i);
        }
    }
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) { return b->cells[a] > b->cells[c]; });
    std::vector<BatchTask1d> tasks;
    std::vector<int> items_of(b->tiles_of);
    for (int i : order) {
        const int nseg = cdiv(b->params[i].nx, mc::kTile);
        for (int s0 = 0; s0 < nseg; s0 += segs) {
            tasks.push_back({i, s0, std::min(segs, nseg - s0), 0});
            items_of[i] += 1;
        }
    }
    MCB_CUDA(cudaMemcpy(b->d_items_of, items_of.data(), sizeof(int) * items_of.size(), cudaMemcpyHostToDevice),
             "items per problem");
    cudaFree(b->d_tasks1d);
    b->d_tasks1d = nullptr;
    b->ntasks1d = (int)tasks.size();
    if (!tasks.empty()) {
        MCB_CUDA(cudaMalloc(&b->d_tasks1d, sizeof(BatchTask1d) * tasks.size()), "tasks");
        MCB_CUDA(cudaMemcpy(b->d_tasks1d, tasks.data(), sizeof(BatchTask1d) * tasks.size(), cudaMemcpyHostToDevice),
                 "tasks");
    }
    b->tasks_segs = segs;
    return MC_OK;
}

// Bind every problem's parameters to `pool` for each stage of the plan:
// state pointers (input, step-start state, output), the stage combination
// and the last-stage flag, so that the kernels read them in place.
mc_status bind_stages(mc_batch* b, const double* pool) {
    if (b->stage_pool == pool) {
        return MC_OK;
    }
    const double* bases[3] = {pool, b->buf_a, b->buf_b};
    const Plan pl = plan_for(b->scheme.time_stepper);
    std::vector<StageParams> tab((size_t)pl.n * b->n);
    for (int st = 0; st < pl.n; ++st) {
        for (int i = 0; i < b->n; ++i) {
            StageParams q = b->params[i];
            const int64_t off = b->problems[i].offset;
            q.q_in = bases[pl.in[st]] + off;
            q.q_old = pool + off;
            q.q_out = const_cast<double*>(bases[pl.out[st]]) + off;
            q.combo = pl.combo[st];
            q.last = st == pl.n - 1;
            q.reset_min = 0;
            tab[(size_t)st * b->n + i] = q;
        }
    }
    // earlier steps on the batch's stream may still read the old binding
    MCB_CUDA(cudaStreamSynchronize(b->stream), "sync");
    MCB_CUDA(cudaMemcpy(b->d_stage, tab.data(), sizeof(StageParams) * tab.size(), cudaMemcpyHostToDevice),
             "stage parameters");
    b->stage_pool = pool;
    return MC_OK;
}

BatchStageParams stage_params(const mc_batch* b, int part, int st, int dynamic, int* counter) {
    BatchStageParams bp;
    std::memset(&bp, 0, sizeof(bp));
    bp.probs = b->d_stage + (size_t)st * b->n;
    bp.items2d = b->d_items2d;
    bp.n2d = b->n2d;
    bp.tasks1d = b->d_tasks1d;
    bp.ntasks1d = b->ntasks1d;
    const int bundles = cdiv(b->ntasks1d, part == mc::kPart1d ? mc::batch_warps<mc::kPart1d>()
                                                                : mc::batch_warps<mc::kPartAll>());
    bp.n_items = part == mc::kPart2d ? b->n2d : part == mc::kPart1d ? bundles : b->n2d + bundles;
    bp.dynamic = dynamic;
    bp.counter = counter;
    bp.items_of = b->d_items_of;
    bp.finished = b->d_finished + (size_t)st * b->n;
    return bp;
}

// Enqueue one full step of the batch on stream s: the stage launches and
// the clock launch.
mc_status enqueue_step(mc_batch* b, double* pool, cudaStream_t s) {
    const Plan pl = plan_for(b->scheme.time_stepper);
    for (int st = 0; st < pl.n; ++st) {
        if (b->merged) {
            const BatchStageParams bp = stage_params(b, mc::kPartAll, st, b->dynamic_all, b->d_counters + 2 * st);
            MCB_CUDA(launch_stage(b, bp, mc::kPartAll, b->grid_all, s, nullptr), "batch stage");
            continue;
        }
        if (b->n2d > 0) {
            const BatchStageParams bp = stage_params(b, mc::kPart2d, st, b->dynamic, b->d_counters + 2 * st);
            MCB_CUDA(launch_stage(b, bp, mc::kPart2d, b->grid, s, nullptr), "batch stage");
        }
        if (b->ntasks1d > 0) {
            const BatchStageParams bp = stage_params(b, mc::kPart1d, st, b->dynamic1d, b->d_counters + 2 * st + 1);
            MCB_CUDA(launch_stage(b, bp, mc::kPart1d, b->grid1d, s, nullptr), "batch stage");
        }
    }
    batch_clock_kernel<<<cdiv(b->n, 256), 256, 0, s>>>(b->d_blocks, b->n, 0, b->d_counters, b->d_finished);
    MCB_CUDA(cudaGetLastError(), "batch clock");
    return MC_OK;
}

mc_status init_clocks(mc_batch* b, double* pool, cudaStream_t s) {
    std::vector<DeviceBlock> blk(b->n);
    for (int i = 0; i < b->n; ++i) {
        DeviceBlock& d = blk[i];
        std::memset(&d, 0, sizeof(d));
        const mc_clock& c = b->problems[i].clock;
        d.cfl_min_bits = mc::kInfBits;
        d.time = c.time;
        d.max_time = c.max_time;
        d.prev_output_time = c.prev_output_time;
        d.output_delta = c.output_delta;
        d.max_cfl = b->problems[i].max_cfl;
        d.done = c.time < c.max_time ? 0 : 1;
    }
    MCB_CUDA(cudaMemcpyAsync(b->d_blocks, blk.data(), sizeof(DeviceBlock) * b->n, cudaMemcpyHostToDevice, s),
             "clocks");
    batch_cfl_kernel<<<b->n, 256, 0, s>>>(b->d_params, b->d_offsets, pool);
    MCB_CUDA(cudaGetLastError(), "batch cfl");
    batch_clock_kernel<<<cdiv(b->n, 256), 256, 0, s>>>(b->d_blocks, b->n, 1, b->d_counters, b->d_finished);
    MCB_CUDA(cudaGetLastError(), "batch clock");
    MCB_CUDA(cudaStreamSynchronize(s), "sync");  // blk must outlive the copy
    b->clocks_ready = true;
    b->clocks_pool = pool;
    return MC_OK;
}

mc_status ensure_graph(mc_batch* b, double* pool) {
    const int key[8] = {b->grid, b->dynamic, b->segs, b->grid1d, b->dynamic1d, b->merged ? 1 : 0, b->grid_all,
                        b->dynamic_all};
    if (b->graph && b->graph_pool == pool && std::equal(key, key + 8, b->graph_key)) {
        return MC_OK;
    }
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    if (mc_status st = build_tasks(b, b->segs)) {
        return st;
    }
    if (mc_status st = bind_stages(b, pool)) {
        return st;
    }
    // kernel attributes are set outside the capture
    for (int part : {mc::kPart2d, mc::kPart1d, mc::kPartAll}) {
        int occ = 0;
        const BatchStageParams probe = stage_params(b, part, 0, 0, b->d_counters);
        MCB_CUDA(launch_stage(b, probe, part, 1, b->stream, &occ), "occupancy");
    }
    cudaGraph_t g = nullptr;
    MCB_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "capture");
    mc_status st = enqueue_step(b, pool, b->stream);
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (st != MC_OK) {
        if (g) {
            cudaGraphDestroy(g);
        }
        return st;
    }
    MCB_CUDA(e, "end capture");
    e = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    MCB_CUDA(e, "instantiate");
    b->graph_pool = pool;
    std::copy(key, key + 8, b->graph_key);
    return MC_OK;
}

} // namespace

extern "C" {

mc_status mc_batch_create(const mc_batch_problem* problems, int32_t n, const mc_scheme* scheme, int64_t pool_doubles,
                          mc_batch** out) {
    if (!problems || !scheme || !out || n <= 0) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null argument or empty batch");
    }
    *out = nullptr;
    const mc_scheme& s = *scheme;
    if (s.reconstruction < 0 || s.reconstruction > 3 || s.slope_limiter < 0 || s.slope_limiter > 2 ||
        s.riemann_solver < 0 || s.riemann_solver > 2 || s.time_stepper < 0 || s.time_stepper > 2 ||
        s.precision < 0 || s.precision > 1 || !std::isfinite(s.gamma)) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "scheme out of range");
    }
    for (int i = 0; i < n; ++i) {
        if (mc_status st = validate_problem(problems[i], s, pool_doubles)) {
            return st;
        }
    }
    mc_batch* b = new (std::nothrow) mc_batch();
    if (!b) {
        return bfail(MC_ERR_OUT_OF_MEMORY, "host allocation");
    }
    b->n = n;
    b->scheme = s;
    b->pool_doubles = pool_doubles;
    b->problems.assign(problems, problems + n);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaSuccess;
    auto alloc = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) {
            e = cudaMalloc(p, bytes);
        }
    };
    alloc((void**)&b->buf_a, sizeof(double) * (size_t)pool_doubles);
    alloc((void**)&b->buf_b, sizeof(double) * (size_t)pool_doubles);
    alloc((void**)&b->d_params, sizeof(StageParams) * n);
    alloc((void**)&b->d_offsets, sizeof(long long) * n);
    alloc((void**)&b->d_stage, sizeof(StageParams) * 4 * (size_t)n);
    alloc((void**)&b->d_blocks, sizeof(DeviceBlock) * n);
    alloc((void**)&b->d_counters, sizeof(int) * kCounters);
    alloc((void**)&b->d_finished, sizeof(int) * 4 * (size_t)n);
    alloc((void**)&b->d_items_of, sizeof(int) * (size_t)n);
    if (e == cudaSuccess) {
        e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    }
    if (e == cudaSuccess) {
        e = cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming);
    }
    if (e == cudaSuccess) {
        e = cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        mc_batch_destroy(b);
        return e == cudaErrorMemoryAllocation ? bfail(MC_ERR_OUT_OF_MEMORY, "device allocation")
                                              : bcuda(e, "mc_batch_create");
    }
    // per-problem parameters (state pointers are bound per launch)
    b->params.resize(n);
    b->cells.resize(n);
    std::vector<long long> offs(n);
    std::vector<BatchItem2d> items;
    std::vector<int> order2d;
    for (int i = 0; i < n; ++i) {
        const mc_grid& g = problems[i].grid;
        StageParams& p = b->params[i];
        std::memset(&p, 0, sizeof(p));
        p.xc = g.xc;
        p.yc = g.yc;
        p.zc = 1;
        p.ng = g.ng;
        p.nx = g.xc - 2 * g.ng;
        p.ny = g.num_dim > 1 ? g.yc - 2 * g.ng : 1;
        p.nz = 1;
        p.nvar = 2 + g.num_dim;
        p.ntracer = 0;
        p.plane = (long long)g.xc * g.yc;
        p.dx = g.dx;
        p.gamma = s.gamma;
        p.dt_dev = &b->d_blocks[i].dt;
        p.blk = &b->d_blocks[i];
        for (int f = 0; f < 6; ++f) {
            p.bc.kind[f] = f < 2 * g.num_dim ? g.bc[f] : MC_BC_USERFN;
        }
        offs[i] = problems[i].offset;
        b->cells[i] = p.plane;
        if (g.num_dim == 2) {
            order2d.push_back(i);
        }
    }
    std::stable_sort(order2d.begin(), order2d.end(), [&](int a, int c) { return b->cells[a] > b->cells[c]; });
    b->tiles_of.assign(n, 0);
    for (int i : order2d) {
        const StageParams& p = b->params[i];
        for (int by = 0; by < cdiv(p.ny, mc::kTile); ++by) {
            for (int bx = 0; bx < cdiv(p.nx, mc::kTile); ++bx) {
                items.push_back({i, bx, by, 0});
                b->tiles_of[i] += 1;
            }
        }
    }
    b->n2d = (int)items.size();
    if (!items.empty()) {
        e = cudaMalloc(&b->d_items2d, sizeof(BatchItem2d) * items.size());
        if (e == cudaSuccess) {
            e = cudaMemcpy(b->d_items2d, items.data(), sizeof(BatchItem2d) * items.size(), cudaMemcpyHostToDevice);
        }
    }
    if (e == cudaSuccess) {
        e = cudaMemcpy(b->d_params, b->params.data(), sizeof(StageParams) * n, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) {
        e = cudaMemcpy(b->d_offsets, offs.data(), sizeof(long long) * n, cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) {
        e = cudaMemset(b->d_counters, 0, sizeof(int) * kCounters);
    }
    if (e == cudaSuccess) {
        e = cudaMemset(b->d_finished, 0, sizeof(int) * 4 * (size_t)n);
    }
    if (e != cudaSuccess) {
        mc_batch_destroy(b);
        return bcuda(e, "mc_batch_create");
    }
    if (mc_status st = build_tasks(b, b->segs)) {
        mc_batch_destroy(b);
        return st;
    }
    int occ[3] = {0, 0, 0};
    for (int part : {mc::kPart2d, mc::kPart1d, mc::kPartAll}) {
        const BatchStageParams probe = stage_params(b, part, 0, 0, b->d_counters);
        e = launch_stage(b, probe, part, 1, b->stream, &occ[part]);
        if (e != cudaSuccess) {
            mc_batch_destroy(b);
            return bcuda(e, "occupancy");
        }
    }
    b->occupancy = std::max(occ[mc::kPart2d], 1);
    b->occupancy1d = std::max(occ[mc::kPart1d], 1);
    b->occupancy_all = std::max(occ[mc::kPartAll], 1);
    b->grid = b->sms * b->occupancy;
    b->grid1d = b->sms * b->occupancy1d;
    b->grid_all = b->sms * b->occupancy_all;
    *out = b;
    return MC_OK;
}

mc_status mc_batch_destroy(mc_batch* b) {
    if (!b) {
        return MC_OK;
    }
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
    }
    cudaFree(b->buf_a);
    cudaFree(b->buf_b);
    cudaFree(b->d_params);
    cudaFree(b->d_offsets);
    cudaFree(b->d_stage);
    cudaFree(b->d_blocks);
    cudaFree(b->d_counters);
    cudaFree(b->d_finished);
    cudaFree(b->d_items_of);
    cudaFree(b->d_items2d);
    cudaFree(b->d_tasks1d);
    if (b->ev_in) {
        cudaEventDestroy(b->ev_in);
    }
    if (b->ev_out) {
        cudaEventDestroy(b->ev_out);
    }
    if (b->stream) {
        cudaStreamDestroy(b->stream);
    }
    delete b;
    return MC_OK;
}

mc_status mc_batch_fill_bcs(mc_batch* b, double* pool, void* stream) {
    if (!b || !pool) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    for (int i = 0; i < b->n; ++i) {
        StageParams p = b->params[i];
        p.q_in = pool + b->problems[i].offset;
        p.q_out = pool + b->problems[i].offset;
        MCB_CUDA(mc::launch_fill_bcs(p, b->problems[i].grid.num_dim, s), "fill_bcs");
    }
    b->clocks_ready = false;  // the state changed: first dt from it again
    return MC_OK;
}

mc_status mc_batch_tune(mc_batch* b, double* pool, void* stream) {
    if (!b || !pool) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    MCB_CUDA(cudaStreamSynchronize(s), "sync");
    if (!b->clocks_ready || b->clocks_pool != pool) {
        if (mc_status st = init_clocks(b, pool, b->stream)) {
            return st;
        }
    }
    if (mc_status st = bind_stages(b, pool)) {
        return st;
    }
    cudaEvent_t t0, t1;
    MCB_CUDA(cudaEventCreate(&t0), "event");
    MCB_CUDA(cudaEventCreate(&t1), "event");
    // time one launch of `part` (stage 0: reads the pool, writes buffer A
    // only), best of three
    auto time_part = [&](int part, int grid, int dyn, float* out) -> mc_status {
        float tmin = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {
            MCB_CUDA(cudaMemsetAsync(b->d_counters, 0, sizeof(int) * kCounters, b->stream), "counters");
            MCB_CUDA(cudaMemsetAsync(b->d_finished, 0, sizeof(int) * 4 * (size_t)b->n, b->stream), "counters");
            const BatchStageParams bp = stage_params(b, part, 0, dyn, b->d_counters);
            MCB_CUDA(cudaEventRecord(t0, b->stream), "event");
            MCB_CUDA(launch_stage(b, bp, part, grid, b->stream, nullptr), "tune launch");
            MCB_CUDA(cudaEventRecord(t1, b->stream), "event");
            MCB_CUDA(cudaEventSynchronize(t1), "event");
            float ms = 0.f;
            MCB_CUDA(cudaEventElapsedTime(&ms, t0, t1), "event");
            tmin = std::min(tmin, ms);
        }
        *out = tmin;
        return MC_OK;
    };
    // candidate grids: 1, 2 or 4 waves of resident CTAs, or one CTA per work
    // item (-1: a plain, non-persistent launch, static only)
    auto sweep = [&](int part, int occ, int n_items, int* best_grid, int* best_dyn, float* best) -> mc_status {
        const int grids[4] = {b->sms * occ, 2 * b->sms * occ, 4 * b->sms * occ, -1};
        for (int gi = 0; gi < 4; ++gi) {
            for (int dyn = 0; dyn < 2; ++dyn) {
                if (grids[gi] < 0 && dyn) {
                    continue;
                }
                const int grid = grids[gi] > 0 ? std::min(grids[gi], n_items) : n_items;
                float ms = 0.f;
                if (mc_status st = time_part(part, grid, dyn, &ms)) {
                    return st;
                }
                if (ms < *best) {
                    *best = ms;
                    *best_grid = grid;
                    *best_dyn = dyn;
                }
            }
        }
        return MC_OK;
    };
    // the two-launch form: each launch on its own
    float split = 0.f;
    if (b->n2d > 0) {
        float best = 1e30f;
        if (mc_status st = sweep(mc::kPart2d, b->occupancy, b->n2d, &b->grid, &b->dynamic, &best)) {
            return st;
        }
        split += best;
    }
    int split_segs = b->segs;
    if (b->ntasks1d > 0) {
        float best = 1e30f;
        for (int so : {1, 2, 4}) {
            if (mc_status st = build_tasks(b, so)) {
                return st;
            }
            const float before = best;
            if (mc_status st = sweep(mc::kPart1d, b->occupancy1d, cdiv(b->ntasks1d, mc::batch_warps<mc::kPart1d>()),
                                     &b->grid1d, &b->dynamic1d, &best)) {
                return st;
            }
            if (best < before) {
                split_segs = so;
            }
        }
        split += best;
    }
    // the one-launch form over both lists
    float all = 1e30f;
    int all_segs = b->segs;
    for (int so : {1, 2, 4}) {
        if (b->ntasks1d == 0 && so != 1) {
            break;
        }
        if (mc_status st = build_tasks(b, so)) {
            return st;
        }
        const float before = all;
        const int n_items = b->n2d + cdiv(b->ntasks1d, mc::batch_warps<mc::kPartAll>());
        if (mc_status st = sweep(mc::kPartAll, b->occupancy_all, n_items, &b->grid_all, &b->dynamic_all, &all)) {
            return st;
        }
        if (all < before) {
            all_segs = so;
        }
    }
    // one launch per stage unless the split form is more than 5 % faster
    // (on the 4096-problem set it measures 2 % faster in FP64 and 0.9 % in
    // FP32: the merged kernel's tile body spills a little more)
    b->merged = all <= 1.05f * split;
    b->segs = b->merged ? all_segs : split_segs;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    MCB_CUDA(cudaMemsetAsync(b->d_counters, 0, sizeof(int) * kCounters, b->stream), "counters");
    MCB_CUDA(cudaMemsetAsync(b->d_finished, 0, sizeof(int) * 4 * (size_t)b->n, b->stream), "counters");
    MCB_CUDA(cudaStreamSynchronize(b->stream), "sync");
    return build_tasks(b, b->segs);
}

mc_status mc_batch_advance(mc_batch* b, double* pool, int64_t steps, void* stream) {
    if (!b || !pool || steps < 0) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null argument or negative steps");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    MCB_CUDA(cudaEventRecord(b->ev_in, s), "event");
    MCB_CUDA(cudaStreamWaitEvent(b->stream, b->ev_in, 0), "wait");
    if (!b->clocks_ready || b->clocks_pool != pool) {
        if (mc_status st = init_clocks(b, pool, b->stream)) {
            return st;
        }
    }
    if (mc_status st = ensure_graph(b, pool)) {
        return st;
    }
    for (int64_t k = 0; k < steps; ++k) {
        MCB_CUDA(cudaGraphLaunch(b->graph, b->stream), "graph launch");
    }
    MCB_CUDA(cudaEventRecord(b->ev_out, b->stream), "event");
    MCB_CUDA(cudaStreamWaitEvent(s, b->ev_out, 0), "wait");
    return MC_OK;
}

mc_status mc_batch_clocks(mc_batch* b, mc_clock* clocks, int64_t* steps, uint32_t* status, void* stream) {
    if (!b) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null batch");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    MCB_CUDA(cudaStreamSynchronize(s), "sync");
    MCB_CUDA(cudaStreamSynchronize(b->stream), "sync");
    std::vector<DeviceBlock> blk(b->n);
    if (b->clocks_ready) {
        MCB_CUDA(cudaMemcpy(blk.data(), b->d_blocks, sizeof(DeviceBlock) * b->n, cudaMemcpyDeviceToHost), "clocks");
    }
    for (int i = 0; i < b->n; ++i) {
        const mc_clock& c0 = b->problems[i].clock;
        if (clocks) {
            clocks[i] = c0;
            if (b->clocks_ready) {
                clocks[i].time = blk[i].time;
                clocks[i].prev_output_time = blk[i].prev_output_time;
            }
        }
        if (steps) {
            steps[i] = b->clocks_ready ? blk[i].steps : 0;
        }
        if (status) {
            status[i] = b->clocks_ready ? blk[i].status : 0;
        }
    }
    return MC_OK;
}

mc_status mc_batch_schedule(const mc_batch* b, int32_t* grid, int32_t* dynamic, int32_t* segs_per_task) {
    if (!b) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null batch");
    }
    if (grid) {
        *grid = b->merged ? b->grid_all : b->grid;
    }
    if (dynamic) {
        *dynamic = b->merged ? b->dynamic_all : b->dynamic;
    }
    if (segs_per_task) {
        *segs_per_task = b->segs;
    }
    return MC_OK;
}

mc_status mc_batch_set_stage_launches(mc_batch* b, int32_t launches) {
    if (!b || (launches != 1 && launches != 2)) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null batch or launches per stage not 1 or 2");
    }
    b->merged = launches == 1;
    return MC_OK;
}

mc_status mc_batch_stage_launches(const mc_batch* b, int32_t* launches) {
    if (!b || !launches) {
        return bfail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    *launches = b->merged ? 1 : 2;
    return MC_OK;
}

} // extern "C"
