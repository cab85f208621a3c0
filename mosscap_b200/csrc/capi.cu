// C ABI of the library (include/mosscap_b200.h): context management, stage
// sequencing of the SSPRK drivers and the device-driven main loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "eos.h"
#include "launch.h"
#include "mosscap_b200.h"
#include "slab.h"

using mc::StageParams;

struct mc_ctx {
    mc_grid grid;
    mc_scheme scheme;
    int device = 0;
    int nx = 1, ny = 1, nz = 1, nvar = 0;
    long long plane = 0;          // cells per variable, ghosts included
    size_t state_bytes = 0;
    double* buf_a = nullptr;      // stage buffers
    double* buf_b = nullptr;
    double* dqxy = nullptr;       // 3D x+y divergence
    mc::DeviceBlock* blk = nullptr;
    mc::DeviceBlock* blk_host = nullptr;  // pinned mirror for read-back
    double* dt_log = nullptr;     // device dt log of mc_advance
    int64_t dt_log_cap = 0;
    int64_t launches = 0;
    bool min_from_clock = false;  // last CFL minimum sits in blk->last_cfl_min
    void (*user_bc)(void*, double*, void*) = nullptr;
    void* user_bc_data = nullptr;
    void (*cfl_hook)(void*, uint64_t*, void*) = nullptr;  // mc_set_cfl_reduce_hook
    void* cfl_hook_data = nullptr;
    mc::SlabExchange* slab = nullptr;  // mc_set_slab_decomposition
    int slab_faces = 0;                // faces whose ghosts the slab exchange fills
    // 2D slabs: the exchange of a stage's border layers overlaps its interior
    // tiles (mc_set_slab_overlap). Border tile rows [0, ov_b0) and
    // [ov_b1, ov_rows) read ghost rows or write layers that are sent; they run
    // on ov_border, their exchange on ov_comm, the interior rows on
    // ov_interior, ordered by events; the caller's stream forks and joins.
    bool slab_overlap = true;
    int ov_b0 = 0, ov_b1 = 0, ov_rows = 0;
    cudaStream_t ov_border = nullptr, ov_interior = nullptr, ov_comm = nullptr;
    cudaEvent_t ov_fork = nullptr;
    cudaEvent_t ov_border_done[4] = {}, ov_interior_done[4] = {}, ov_exch_done[4] = {};
    // mc_step_host: copy streams and events of its pipeline (created on first use)
    cudaStream_t hs_in = nullptr, hs_out = nullptr;
    cudaEvent_t hs_fork = nullptr, hs_join = nullptr;
    cudaEvent_t hs_ev_in[16] = {}, hs_ev_out[16] = {};
    int gravity = 0;              // mc_set_gravity
    double grav[3] = {0.0, 0.0, 0.0};
    // non-ideal EOS (mc_set_eos)
    int eos_type = 0;
    int eos_ion = 0;
    double eos_avg_mass = 1.0;
    double* eos_y = nullptr;      // y_space, T_space (device, plane each)
    double* eos_T = nullptr;
    double* eos_ytab = nullptr;   // tabulated: tables (device) and grid
    double* eos_lTtab = nullptr;
    double tab_x0 = 0.0, tab_dx = 1.0, tab_y0 = 0.0, tab_dy = 1.0;
    int tab_nx = 0, tab_ny = 0;
    double* buf_eos = nullptr;    // tabulated: the first stage's shifted input
    const double* last_stage_in = nullptr;  // input of the last stage of the latest step
    // kernel timing (mc_profile_stages)
    bool profiling = false;
    struct Timed {
        cudaEvent_t start, stop;
        int kind;
        // an overlapped stage's second piece (null otherwise): the stage
        // lasts from the first start to the last stop
        cudaEvent_t start2, stop2;
    };
    std::vector<Timed> timed;
    std::vector<cudaEvent_t> event_pool;
};

namespace {

thread_local std::string g_error;

mc_status fail(mc_status s, const std::string& msg) {
    g_error = msg;
    return s;
}

mc_status cuda_fail(cudaError_t e, const char* where) {
    return fail(MC_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define MC_CUDA(call, where)                   \
    do {                                       \
        cudaError_t e_ = (call);               \
        if (e_ != cudaSuccess) {               \
            return cuda_fail(e_, where);       \
        }                                      \
    } while (0)

int halo_needed(int rec) {
    return rec == MC_RECON_FOG ? 1 : rec == MC_RECON_MUSCL ? 2 : 3;
}

StageParams base_params(const mc_ctx* c) {
    StageParams p;
    std::memset(&p, 0, sizeof(p));
    p.xc = c->grid.xc;
    p.yc = c->grid.yc;
    p.zc = c->grid.zc;
    p.ng = c->grid.ng;
    p.nx = c->nx;
    p.ny = c->ny;
    p.nz = c->nz;
    p.nvar = c->nvar;
    p.ntracer = c->grid.num_tracers;
    p.plane = c->plane;
    p.dx = c->grid.dx;
    p.gamma = c->scheme.gamma;
    p.blk = c->blk;
    p.gravity = c->gravity;
    for (int a = 0; a < 3; ++a) {
        p.grav[a] = c->grav[a];
    }
    for (int f = 0; f < 6; ++f) {
        p.bc.kind[f] = c->grid.bc[f];
        for (int v = 0; v < mc::kMaxVars; ++v) {
            p.bc.cval[f][v] = v < 5 ? c->grid.bc_const[f][v] : 0.0;
        }
    }
    return p;
}

cudaEvent_t pooled_event(mc_ctx* c) {
    if (!c->event_pool.empty()) {
        cudaEvent_t e = c->event_pool.back();
        c->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

cudaError_t launch_stage_kernel(mc_ctx* c, const StageParams& p, int pass, cudaStream_t s);

// Launch one stage kernel; with profiling on, bracket it with events.
cudaError_t launch_stage(mc_ctx* c, const StageParams& p, int pass, cudaStream_t s) {
    if (!c->profiling) {
        return launch_stage_kernel(c, p, pass, s);
    }
    mc_ctx::Timed t{pooled_event(c), pooled_event(c), c->grid.num_dim == 3 ? pass : 0, nullptr, nullptr};
    cudaEventRecord(t.start, s);
    const cudaError_t e = launch_stage_kernel(c, p, pass, s);
    cudaEventRecord(t.stop, s);
    c->timed.push_back(t);
    return e;
}

cudaError_t launch_stage_kernel(mc_ctx* c, const StageParams& p, int pass, cudaStream_t s) {
    const int nd = c->grid.num_dim;
    const bool f32 = c->scheme.precision == MC_PRECISION_FP32_COMPENSATED;
    const int r = c->scheme.reconstruction, l = c->scheme.slope_limiter, rs = c->scheme.riemann_solver;
    c->launches += 1;
    if (nd == 2 && pass == 0 && p.dqxy) {
        // the deferred form (mc_step_host)
        if (p.gravity) {
            return f32 ? mc::launch_stage_d2_fp32_src_defer(p, r, l, rs, pass, s)
                       : mc::launch_stage_d2_fp64_src_defer(p, r, l, rs, pass, s);
        }
        return f32 ? mc::launch_stage_d2_fp32_defer(p, r, l, rs, pass, s)
                   : mc::launch_stage_d2_fp64_defer(p, r, l, rs, pass, s);
    }
    if (p.gravity) {
        if (nd == 1) {
            return f32 ? mc::launch_stage_d1_fp32_src(p, r, l, rs, pass, s)
                       : mc::launch_stage_d1_fp64_src(p, r, l, rs, pass, s);
        }
        if (nd == 2) {
            return f32 ? mc::launch_stage_d2_fp32_src(p, r, l, rs, pass, s)
                       : mc::launch_stage_d2_fp64_src(p, r, l, rs, pass, s);
        }
        return f32 ? mc::launch_stage_d3_fp32_src(p, r, l, rs, pass, s)
                   : mc::launch_stage_d3_fp64_src(p, r, l, rs, pass, s);
    }
    if (nd == 1) {
        return f32 ? mc::launch_stage_d1_fp32(p, r, l, rs, pass, s) : mc::launch_stage_d1_fp64(p, r, l, rs, pass, s);
    }
    if (nd == 2) {
        return f32 ? mc::launch_stage_d2_fp32(p, r, l, rs, pass, s) : mc::launch_stage_d2_fp64(p, r, l, rs, pass, s);
    }
    return f32 ? mc::launch_stage_d3_fp32(p, r, l, rs, pass, s) : mc::launch_stage_d3_fp64(p, r, l, rs, pass, s);
}

mc::EosLaunch eos_launch(const mc_ctx* c, const double* q_in, double* q_out, bool skip_when_done) {
    mc::EosLaunch L;
    std::memset(&L, 0, sizeof(L));
    L.type = c->eos_type;
    L.q_in = q_in;
    L.q_out = q_out;
    L.y = c->eos_y;
    L.T = c->eos_T;
    L.plane = c->plane;
    L.nvar = c->nvar;
    L.gamma = c->scheme.gamma;
    L.avg_mass = c->eos_avg_mass;
    L.ionisation_e = c->eos_ion;
    L.x_start = c->tab_x0;
    L.x_step = c->tab_dx;
    L.y_start = c->tab_y0;
    L.y_step = c->tab_dy;
    L.nx_tab = c->tab_nx;
    L.ny_tab = c->tab_ny;
    L.y_table = c->eos_ytab;
    L.log_T_table = c->eos_lTtab;
    L.blk = c->blk;
    L.skip_when_done = skip_when_done ? 1 : 0;
    return L;
}

// Faces of kind MC_BC_USERFN among the active ones (bit f = face f) whose
// ghosts the caller's hook fills (not the slab exchange).
int user_face_mask(const mc_ctx* c) {
    int m = 0;
    for (int f = 0; f < 2 * c->grid.num_dim; ++f) {
        if (c->grid.bc[f] == MC_BC_USERFN && !((c->slab_faces >> f) & 1)) {
            m |= 1 << f;
        }
    }
    return m;
}

// The slab exchange of Q's ghost layers, if the context is one slab of a
// decomposed problem.
mc_status exchange_slab(mc_ctx* c, double* q, cudaStream_t s) {
    if (!c->slab) {
        return MC_OK;
    }
    const char* why = "";
    if (mc::slab_exchange(c->slab, q, s, &why) != cudaSuccess) {
        return fail(MC_ERR_CUDA, std::string("slab exchange: ") + why);
    }
    return MC_OK;
}

mc_status enqueue_step_overlapped(mc_ctx* c, double* Q, double dt, const double* dt_dev, bool reset_min,
                                  cudaStream_t s);
bool overlapped(const mc_ctx* c);

// Enqueue one SSPRK step on Q. dt_dev (device-driven loop) or dt (host).
mc_status enqueue_step(mc_ctx* c, double* Q, double dt, const double* dt_dev, bool reset_min, cudaStream_t s) {
    if (overlapped(c)) {
        return enqueue_step_overlapped(c, Q, dt, dt_dev, reset_min, s);
    }
    const mc::StagePlan plan = mc::plan_for(c->scheme.time_stepper);
    double* bufs[3] = {Q, c->buf_a, c->buf_b};
    c->last_stage_in = bufs[plan.in[plan.n - 1]];
    for (int st = 0; st < plan.n; ++st) {
        StageParams p = base_params(c);
        p.q_in = bufs[plan.in[st]];
        p.q_old = Q;
        p.q_out = bufs[plan.out[st]];
        p.dqxy = c->dqxy;
        p.dt = dt;
        p.dt_dev = dt_dev;
        p.combo = plan.combo[st];
        p.last = st == plan.n - 1;
        p.reset_min = (reset_min && st == 0) ? 1 : 0;
        if (c->eos_type != mc::kEosIdeal) {
            // update_eos ahead of the sweep; the tabulated kind shifts the
            // energy, which for the first stage goes to a copy so that the
            // step-start state keeps its own
            double* q_eos = const_cast<double*>(p.q_in);
            if (c->eos_type == mc::kEosTabulated && p.q_in == Q) {
                q_eos = c->buf_eos;
                p.q_in = q_eos;
            }
            c->launches += 1;
            MC_CUDA(mc::launch_eos_update(eos_launch(c, bufs[plan.in[st]], q_eos, dt_dev != nullptr),
                                          c->grid.num_dim, s),
                    "EOS update");
        }
        MC_CUDA(launch_stage(c, p, 0, s), "stage launch");
        if (c->grid.num_dim == 3) {
            p.reset_min = 0;
            MC_CUDA(launch_stage(c, p, 1, s), "stage launch (z pass)");
        }
        if (mc_status st = exchange_slab(c, p.q_out, s)) {
            return st;
        }
        if (c->user_bc) {
            c->user_bc(c->user_bc_data, p.q_out, (void*)s);
            // the hook fills the MC_BC_USERFN ghosts after the fused CFL
            // reduction of the last stage; add their layers to it
            const int mask = user_face_mask(c);
            if (p.last && mask) {
                StageParams g = p;
                g.q_in = p.q_out;
                c->launches += 1;
                MC_CUDA(mc::launch_cfl_min_ghosts(g, c->grid.num_dim, mask, s), "cfl_min (user ghosts)");
            }
        }
    }
    return MC_OK;
}

// Whether a step of this context runs with the slab exchange overlapping
// the interior tiles.
bool overlapped(const mc_ctx* c) {
    return c->slab && c->slab_overlap && c->ov_border && c->grid.num_dim == 2 && c->eos_type == mc::kEosIdeal &&
           !c->user_bc && c->ov_b0 < c->ov_b1;
}

// One SSPRK step of a 2D slab with each stage's exchange beside its
// interior tiles. Per stage: the border tile rows (after the previous stage
// and its exchange) on ov_border; the exchange of the layers they wrote on
// ov_comm; the interior tile rows (after the previous stage's border rows;
// its interior rows come earlier on the same stream) on ov_interior. The
// interior rows neither read ghost rows nor write the layers that are sent,
// and the exchange writes only ghost rows, so the pieces touch disjoint
// cells; the result is that of enqueue_step. The caller's stream waits for
// the last stage and its exchange.
mc_status enqueue_step_overlapped(mc_ctx* c, double* Q, double dt, const double* dt_dev, bool reset_min,
                                  cudaStream_t s) {
    const mc::StagePlan plan = mc::plan_for(c->scheme.time_stepper);
    double* bufs[3] = {Q, c->buf_a, c->buf_b};
    c->last_stage_in = bufs[plan.in[plan.n - 1]];
    MC_CUDA(cudaEventRecord(c->ov_fork, s), "fork");
    MC_CUDA(cudaStreamWaitEvent(c->ov_border, c->ov_fork, 0), "fork");
    MC_CUDA(cudaStreamWaitEvent(c->ov_interior, c->ov_fork, 0), "fork");
    MC_CUDA(cudaStreamWaitEvent(c->ov_comm, c->ov_fork, 0), "fork");
    for (int st = 0; st < plan.n; ++st) {
        StageParams p = base_params(c);
        p.q_in = bufs[plan.in[st]];
        p.q_old = Q;
        p.q_out = bufs[plan.out[st]];
        p.dt = dt;
        p.dt_dev = dt_dev;
        p.combo = plan.combo[st];
        p.last = st == plan.n - 1;
        // both pieces of the first stage reset the minimum the last stage forms
        p.reset_min = (reset_min && st == 0) ? 1 : 0;
        StageParams pb = p;
        pb.row_split = c->ov_b0;
        pb.row_skip = c->ov_b1 - c->ov_b0;
        pb.tile_rows = c->ov_b0 + (c->ov_rows - c->ov_b1);
        StageParams pi = p;
        pi.row_split = 0;
        pi.row_skip = c->ov_b0;
        pi.tile_rows = c->ov_b1 - c->ov_b0;
        if (st > 0) {
            MC_CUDA(cudaStreamWaitEvent(c->ov_border, c->ov_interior_done[st - 1], 0), "wait");
            MC_CUDA(cudaStreamWaitEvent(c->ov_border, c->ov_exch_done[st - 1], 0), "wait");
            MC_CUDA(cudaStreamWaitEvent(c->ov_interior, c->ov_border_done[st - 1], 0), "wait");
        }
        mc_ctx::Timed t{nullptr, nullptr, 0, nullptr, nullptr};
        if (c->profiling) {
            t = mc_ctx::Timed{pooled_event(c), pooled_event(c), 0, pooled_event(c), pooled_event(c)};
            cudaEventRecord(t.start, c->ov_border);
        }
        MC_CUDA(launch_stage_kernel(c, pb, 0, c->ov_border), "stage launch (border rows)");
        if (c->profiling) {
            cudaEventRecord(t.stop, c->ov_border);
        }
        MC_CUDA(cudaEventRecord(c->ov_border_done[st], c->ov_border), "event");
        MC_CUDA(cudaStreamWaitEvent(c->ov_comm, c->ov_border_done[st], 0), "wait");
        if (mc_status e = exchange_slab(c, p.q_out, c->ov_comm)) {
            return e;
        }
        MC_CUDA(cudaEventRecord(c->ov_exch_done[st], c->ov_comm), "event");
        if (c->profiling) {
            cudaEventRecord(t.start2, c->ov_interior);
        }
        MC_CUDA(launch_stage_kernel(c, pi, 0, c->ov_interior), "stage launch (interior rows)");
        if (c->profiling) {
            cudaEventRecord(t.stop2, c->ov_interior);
            c->timed.push_back(t);
        }
        MC_CUDA(cudaEventRecord(c->ov_interior_done[st], c->ov_interior), "event");
    }
    MC_CUDA(cudaStreamWaitEvent(s, c->ov_interior_done[plan.n - 1], 0), "join");
    MC_CUDA(cudaStreamWaitEvent(s, c->ov_exch_done[plan.n - 1], 0), "join");
    return MC_OK;
}

// ---- mc_step_host ------------------------------------------------------------

constexpr int kHostBands = 16;  // bands of tile rows of the pipelined host step (16: 1.3 % faster than 8 on KH 2048^2)

// Whether mc_step_host overlaps its copies with the step (2D, ideal EOS, no
// hooks or slab exchange, at least two tile rows).
bool host_pipelined(const mc_ctx* c) {
    return c->grid.num_dim == 2 && c->eos_type == mc::kEosIdeal && !c->user_bc && !c->slab && !c->cfl_hook &&
           c->ny > mc::kTile;
}

mc_status create_host_streams(mc_ctx* c) {
    if (c->hs_in) {
        return MC_OK;
    }
    MC_CUDA(cudaStreamCreateWithFlags(&c->hs_in, cudaStreamNonBlocking), "stream");
    MC_CUDA(cudaStreamCreateWithFlags(&c->hs_out, cudaStreamNonBlocking), "stream");
    MC_CUDA(cudaEventCreateWithFlags(&c->hs_fork, cudaEventDisableTiming), "event");
    MC_CUDA(cudaEventCreateWithFlags(&c->hs_join, cudaEventDisableTiming), "event");
    for (int b = 0; b < kHostBands; ++b) {
        MC_CUDA(cudaEventCreateWithFlags(&c->hs_ev_in[b], cudaEventDisableTiming), "event");
        MC_CUDA(cudaEventCreateWithFlags(&c->hs_ev_out[b], cudaEventDisableTiming), "event");
    }
    return MC_OK;
}

void destroy_host_streams(mc_ctx* c) {
    for (cudaStream_t* st : {&c->hs_in, &c->hs_out}) {
        if (*st) {
            cudaStreamSynchronize(*st);
            cudaStreamDestroy(*st);
            *st = nullptr;
        }
    }
    for (cudaEvent_t* e : {&c->hs_fork, &c->hs_join}) {
        if (*e) {
            cudaEventDestroy(*e);
            *e = nullptr;
        }
    }
    for (int b = 0; b < kHostBands; ++b) {
        for (cudaEvent_t* e : {&c->hs_ev_in[b], &c->hs_ev_out[b]}) {
            if (*e) {
                cudaEventDestroy(*e);
                *e = nullptr;
            }
        }
    }
}

// The pipelined host step (2D). The grid's tile rows split into bands.
//  1. The state arrives band by band (rows of all variables, one 2D copy per
//     band) on hs_in; stage 0's tiles of a band run as soon as the rows they
//     read have arrived, writing only their x+y divergence (into buf_b,
//     which no stage before the second reads).
//  2. Once the whole state is in: the CFL minimum and dt (the device clock,
//     the output clamp of compute_dt), then the rest of stage 0 per cell
//     (finish2d_kernel: the same operations the tiles would have done).
//  3. The middle stages whole; the last stage band by band, each band's
//     interior rows copied back on hs_out as soon as it is done (no later
//     band writes them), the ghost rows after the last band.
// Result and dt are those of compute_dt + time_step.
mc_status step_host_pipelined(mc_ctx* c, double* Qh, double* Q, const mc_clock* clk, double* dt_out,
                              cudaStream_t s) {
    if (mc_status st = create_host_streams(c)) {
        return st;
    }
    const mc::StagePlan plan = mc::plan_for(c->scheme.time_stepper);
    double* bufs[3] = {Q, c->buf_a, c->buf_b};
    const int ng = c->grid.ng, ny = c->ny;
    const long long xc = c->grid.xc, yc = c->grid.yc;
    const int rows = (ny + mc::kTile - 1) / mc::kTile;
    const int nb = std::min(kHostBands, rows);
    int t[kHostBands + 1];
    for (int b = 0; b <= nb; ++b) {
        t[b] = (int)((long long)b * rows / nb);
    }
    // padded-row boundaries of the input bands: the first and last also
    // carry the ghost rows
    auto in_row = [&](int b) -> long long { return b == 0 ? 0 : (b == nb ? yc : ng + (long long)t[b] * mc::kTile); };
    const size_t pitch = sizeof(double) * (size_t)c->plane;
    const size_t row_bytes = sizeof(double) * (size_t)xc;
    const int nvar = c->nvar;
    MC_CUDA(cudaEventRecord(c->hs_fork, s), "fork");
    MC_CUDA(cudaStreamWaitEvent(c->hs_in, c->hs_fork, 0), "fork");
    MC_CUDA(cudaStreamWaitEvent(c->hs_out, c->hs_fork, 0), "fork");
    for (int b = 0; b < nb; ++b) {
        const long long r0 = in_row(b), r1 = in_row(b + 1);
        MC_CUDA(cudaMemcpy2DAsync(Q + r0 * xc, pitch, Qh + r0 * xc, pitch, (size_t)(r1 - r0) * row_bytes, nvar,
                                  cudaMemcpyHostToDevice, c->hs_in),
                "state in");
        MC_CUDA(cudaEventRecord(c->hs_ev_in[b], c->hs_in), "event");
    }
    const double inf = std::numeric_limits<double>::infinity();
    MC_CUDA(mc::launch_clock_init(c->blk, clk ? clk->time : 0.0, clk ? clk->max_time : inf,
                                  clk ? clk->prev_output_time : 0.0, clk ? clk->output_delta : inf,
                                  c->scheme.max_cfl, s),
            "clock init");
    // 1. stage 0's divergence, band by band
    StageParams d = base_params(c);
    d.q_in = Q;
    d.q_old = Q;
    d.q_out = bufs[plan.out[0]];
    d.dqxy = c->buf_b;
    d.combo = plan.combo[0];
    for (int b = 0; b < nb; ++b) {
        // the band's tiles read H rows of the next band
        MC_CUDA(cudaStreamWaitEvent(s, c->hs_ev_in[std::min(b + 1, nb - 1)], 0), "wait");
        StageParams pb = d;
        pb.row_skip = t[b];
        pb.tile_rows = t[b + 1] - t[b];
        MC_CUDA(launch_stage_kernel(c, pb, 0, s), "stage 0 divergence");
    }
    // 2. dt, then the rest of stage 0
    StageParams g = base_params(c);
    g.q_in = Q;
    MC_CUDA(mc::launch_cfl_min(g, 2, s), "cfl_min");
    MC_CUDA(mc::launch_clock_advance(c->blk, nullptr, 1, s), "clock");
    c->launches += 3;
    const double* dt_dev = &c->blk->dt;
    StageParams f = d;
    f.dt_dev = dt_dev;
    MC_CUDA(launch_stage_kernel(c, f, 2, s), "stage 0 finish");
    // 3. the other stages; the last one band by band behind the copies
    for (int st = 1; st < plan.n; ++st) {
        StageParams p = base_params(c);
        p.q_in = bufs[plan.in[st]];
        p.q_old = Q;
        p.q_out = bufs[plan.out[st]];
        p.dt_dev = dt_dev;
        p.combo = plan.combo[st];
        p.last = st == plan.n - 1;
        if (!p.last) {
            MC_CUDA(launch_stage_kernel(c, p, 0, s), "stage launch");
            continue;
        }
        for (int b = 0; b < nb; ++b) {
            StageParams pb = p;
            pb.row_skip = t[b];
            pb.tile_rows = t[b + 1] - t[b];
            MC_CUDA(launch_stage_kernel(c, pb, 0, s), "last stage");
            MC_CUDA(cudaEventRecord(c->hs_ev_out[b], s), "event");
            MC_CUDA(cudaStreamWaitEvent(c->hs_out, c->hs_ev_out[b], 0), "wait");
            const long long r0 = ng + (long long)t[b] * mc::kTile;
            const long long r1 = ng + std::min((long long)ny, (long long)t[b + 1] * mc::kTile);
            MC_CUDA(cudaMemcpy2DAsync(Qh + r0 * xc, pitch, Q + r0 * xc, pitch, (size_t)(r1 - r0) * row_bytes, nvar,
                                      cudaMemcpyDeviceToHost, c->hs_out),
                    "state out");
        }
    }
    c->last_stage_in = bufs[plan.in[plan.n - 1]];
    // the ghost rows (the end bands' scatter writes them) and the clock
    MC_CUDA(cudaMemcpy2DAsync(Qh, pitch, Q, pitch, (size_t)ng * row_bytes, nvar, cudaMemcpyDeviceToHost, c->hs_out),
            "ghost rows out");
    MC_CUDA(cudaMemcpy2DAsync(Qh + (ng + (long long)ny) * xc, pitch, Q + (ng + (long long)ny) * xc, pitch,
                              (size_t)ng * row_bytes, nvar, cudaMemcpyDeviceToHost, c->hs_out),
            "ghost rows out");
    MC_CUDA(cudaMemcpyAsync(c->blk_host, c->blk, sizeof(mc::DeviceBlock), cudaMemcpyDeviceToHost, c->hs_out),
            "read-back");
    MC_CUDA(cudaEventRecord(c->hs_join, c->hs_out), "join");
    MC_CUDA(cudaStreamWaitEvent(s, c->hs_join, 0), "join");
    MC_CUDA(cudaStreamSynchronize(s), "sync");
    c->min_from_clock = false;
    const mc::DeviceBlock& k = *c->blk_host;
    *dt_out = k.dt;
    if (k.done) {
        return fail(MC_ERR_INVALID_ARGUMENT, "dt must be positive and finite (the step was not taken)");
    }
    return MC_OK;
}

// The domain-wide reduction of the CFL minimum word: the slab
// decomposition's all-reduce and the caller's hook, if any.
mc_status reduce_cfl(mc_ctx* c, cudaStream_t s) {
    uint64_t* word = reinterpret_cast<uint64_t*>(&c->blk->cfl_min_bits);
    if (c->slab) {
        const char* why = "";
        if (mc::slab_reduce_min(c->slab, word, s, &why) != cudaSuccess) {
            return fail(MC_ERR_CUDA, std::string("slab CFL all-reduce: ") + why);
        }
    }
    if (c->cfl_hook) {
        c->cfl_hook(c->cfl_hook_data, word, (void*)s);
    }
    return MC_OK;
}

double clamp_to_output(double dt, const mc_clock* k) {
    // source/Hydro.cpp:231-241
    const double cand = k->prev_output_time + k->output_delta;
    const double next_write = (cand < k->max_time) ? cand : k->max_time;
    if (k->time + dt >= next_write) {
        dt = next_write - k->time;
        while (k->time + dt < next_write) {
            dt = std::nextafter(dt, DBL_MAX);
        }
    }
    return dt;
}

// Streams, events and border tile rows of the overlapped slab step (2D).
mc_status create_overlap(mc_ctx* c) {
    const int ng = c->grid.ng, ny = c->ny;
    const int rows = (ny + mc::kTile - 1) / mc::kTile;
    // border rows: those whose tiles read ghost rows (first row y0 < H <= ng)
    // or write layers that are sent (y0 < ng, or y1 > ny - ng)
    int b0 = 0;
    while (b0 < rows && b0 * mc::kTile < ng) {
        ++b0;
    }
    int b1 = rows;
    while (b1 > b0 && std::min(ny, b1 * mc::kTile) > ny - ng) {
        --b1;
    }
    c->ov_b0 = b0;
    c->ov_b1 = b1;
    c->ov_rows = rows;
    int least = 0, greatest = 0;
    MC_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest), "stream priorities");
    MC_CUDA(cudaStreamCreateWithPriority(&c->ov_border, cudaStreamNonBlocking, greatest), "stream");
    MC_CUDA(cudaStreamCreateWithPriority(&c->ov_comm, cudaStreamNonBlocking, greatest), "stream");
    MC_CUDA(cudaStreamCreateWithPriority(&c->ov_interior, cudaStreamNonBlocking, least), "stream");
    MC_CUDA(cudaEventCreateWithFlags(&c->ov_fork, cudaEventDisableTiming), "event");
    for (int k = 0; k < 4; ++k) {
        MC_CUDA(cudaEventCreateWithFlags(&c->ov_border_done[k], cudaEventDisableTiming), "event");
        MC_CUDA(cudaEventCreateWithFlags(&c->ov_interior_done[k], cudaEventDisableTiming), "event");
        MC_CUDA(cudaEventCreateWithFlags(&c->ov_exch_done[k], cudaEventDisableTiming), "event");
    }
    return MC_OK;
}

void destroy_overlap(mc_ctx* c) {
    for (cudaStream_t* st : {&c->ov_border, &c->ov_interior, &c->ov_comm}) {
        if (*st) {
            cudaStreamSynchronize(*st);
            cudaStreamDestroy(*st);
            *st = nullptr;
        }
    }
    for (cudaEvent_t* e : {&c->ov_fork}) {
        if (*e) {
            cudaEventDestroy(*e);
            *e = nullptr;
        }
    }
    for (int k = 0; k < 4; ++k) {
        for (cudaEvent_t* e : {&c->ov_border_done[k], &c->ov_interior_done[k], &c->ov_exch_done[k]}) {
            if (*e) {
                cudaEventDestroy(*e);
                *e = nullptr;
            }
        }
    }
}

mc_status check_ctx(const mc_ctx* c) {
    if (!c) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null context");
    }
    return MC_OK;
}

// A MC_BC_USERFN face is filled only by the caller's hook (or the slab
// exchange).
mc_status check_user_bc(const mc_ctx* c) {
    for (int f = 0; f < 2 * c->grid.num_dim; ++f) {
        if (c->grid.bc[f] == MC_BC_USERFN && !((c->slab_faces >> f) & 1) && !c->user_bc) {
            return fail(MC_ERR_INVALID_ARGUMENT, "a MC_BC_USERFN face needs mc_set_user_bc");
        }
    }
    return MC_OK;
}

} // namespace

namespace mc {
void set_last_error(const char* msg) {
    g_error = msg;
}
} // namespace mc

extern "C" {

int32_t mc_abi_version(void) {
    return MC_ABI_VERSION;
}

const char* mc_last_error(void) {
    return g_error.c_str();
}

mc_status mc_create(const mc_grid* grid, const mc_scheme* scheme, mc_ctx** out) {
    if (!grid || !scheme || !out) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    *out = nullptr;
    const mc_grid& g = *grid;
    const mc_scheme& s = *scheme;
    if (g.num_dim < 1 || g.num_dim > 3) {
        return fail(MC_ERR_INVALID_ARGUMENT, "num_dim must be 1, 2 or 3");
    }
    if (s.reconstruction < 0 || s.reconstruction > 3 || s.slope_limiter < 0 || s.slope_limiter > 2 ||
        s.riemann_solver < 0 || s.riemann_solver > 2 || s.time_stepper < 0 || s.time_stepper > 2 ||
        s.precision < 0 || s.precision > 1) {
        return fail(MC_ERR_INVALID_ARGUMENT, "scheme enum out of range");
    }
    if (g.ng < halo_needed(s.reconstruction) || g.ng > mc::kMaxGhost) {
        return fail(MC_ERR_INVALID_ARGUMENT, "ng below the reconstruction's need or above 8");
    }
    const int ext[3] = {g.xc, g.yc, g.zc};
    for (int a = 0; a < 3; ++a) {
        if (a < g.num_dim) {
            if (ext[a] - 2 * g.ng < g.ng) {
                return fail(MC_ERR_INVALID_ARGUMENT, "each active axis needs at least ng interior cells");
            }
        } else if (ext[a] != 1) {
            return fail(MC_ERR_INVALID_ARGUMENT, "inactive axes must have extent 1");
        }
    }
    if (g.num_tracers < 0 || 2 + g.num_dim + g.num_tracers > mc::kMaxVars) {
        return fail(MC_ERR_INVALID_ARGUMENT, "too many variables (at most 8)");
    }
    if (!(g.dx > 0.0) || !std::isfinite(g.dx) || !std::isfinite(s.gamma) || !std::isfinite(s.max_cfl)) {
        return fail(MC_ERR_INVALID_ARGUMENT, "dx, gamma and max_cfl must be finite (dx > 0)");
    }
    for (int f = 0; f < 2 * g.num_dim; ++f) {
        if (g.bc[f] < 0 || g.bc[f] > MC_BC_USERFN) {
            return fail(MC_ERR_INVALID_ARGUMENT, "boundary kind out of range");
        }
        if (g.bc[f] == MC_BC_CONSTANT && 2 + g.num_dim + g.num_tracers > 5) {
            return fail(MC_ERR_UNSUPPORTED, "constant boundaries hold at most 5 variables");
        }
    }
    if ((g.bc[0] == MC_BC_PERIODIC) != (g.bc[1] == MC_BC_PERIODIC) ||
        (g.num_dim > 1 && (g.bc[2] == MC_BC_PERIODIC) != (g.bc[3] == MC_BC_PERIODIC)) ||
        (g.num_dim > 2 && (g.bc[4] == MC_BC_PERIODIC) != (g.bc[5] == MC_BC_PERIODIC))) {
        return fail(MC_ERR_INVALID_ARGUMENT, "periodic boundaries come in pairs");
    }
    mc_ctx* c = new (std::nothrow) mc_ctx();
    if (!c) {
        return fail(MC_ERR_OUT_OF_MEMORY, "host allocation");
    }
    c->grid = g;
    // unused axes: keep their kinds out of the ghost logic
    for (int f = 2 * g.num_dim; f < 6; ++f) {
        c->grid.bc[f] = MC_BC_USERFN;
    }
    c->scheme = s;
    cudaGetDevice(&c->device);
    c->nx = g.xc - 2 * g.ng;
    c->ny = g.num_dim > 1 ? g.yc - 2 * g.ng : 1;
    c->nz = g.num_dim > 2 ? g.zc - 2 * g.ng : 1;
    c->nvar = 2 + g.num_dim + g.num_tracers;
    c->plane = (long long)g.xc * g.yc * g.zc;
    c->state_bytes = sizeof(double) * (size_t)c->nvar * (size_t)c->plane;
    cudaError_t e = cudaMalloc(&c->buf_a, c->state_bytes);
    if (e == cudaSuccess) {
        e = cudaMalloc(&c->buf_b, c->state_bytes);
    }
    if (e == cudaSuccess && g.num_dim == 3) {
        e = cudaMalloc(&c->dqxy, sizeof(double) * (size_t)c->nvar * c->nx * c->ny * c->nz);
    }
    if (e == cudaSuccess) {
        e = cudaMalloc(&c->blk, sizeof(mc::DeviceBlock));
    }
    if (e == cudaSuccess) {
        e = cudaMallocHost(&c->blk_host, sizeof(mc::DeviceBlock));
    }
    if (e == cudaSuccess) {
        e = cudaMemset(c->blk, 0, sizeof(mc::DeviceBlock));
    }
    if (e != cudaSuccess) {
        mc_destroy(c);
        return e == cudaErrorMemoryAllocation ? fail(MC_ERR_OUT_OF_MEMORY, "device allocation")
                                              : cuda_fail(e, "mc_create");
    }
    *out = c;
    return MC_OK;
}

mc_status mc_destroy(mc_ctx* c) {
    if (!c) {
        return MC_OK;
    }
    destroy_overlap(c);  // its streams drained before the communicator goes
    destroy_host_streams(c);
    mc::slab_destroy(c->slab);
    cudaFree(c->buf_a);
    cudaFree(c->buf_b);
    cudaFree(c->dqxy);
    cudaFree(c->blk);
    cudaFree(c->dt_log);
    cudaFree(c->eos_y);
    cudaFree(c->eos_T);
    cudaFree(c->eos_ytab);
    cudaFree(c->eos_lTtab);
    cudaFree(c->buf_eos);
    if (c->blk_host) {
        cudaFreeHost(c->blk_host);
    }
    for (auto& t : c->timed) {
        cudaEventDestroy(t.start);
        cudaEventDestroy(t.stop);
        if (t.start2) {
            cudaEventDestroy(t.start2);
            cudaEventDestroy(t.stop2);
        }
    }
    for (auto e : c->event_pool) {
        cudaEventDestroy(e);
    }
    delete c;
    return MC_OK;
}

mc_status mc_set_user_bc(mc_ctx* c, void (*fn)(void* user, double* Q, void* stream), void* user) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    c->user_bc = fn;
    c->user_bc_data = user;
    return MC_OK;
}

mc_status mc_set_gravity(mc_ctx* c, int32_t enabled, double gx, double gy, double gz) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    c->gravity = enabled ? 1 : 0;
    c->grav[0] = enabled ? gx : 0.0;
    c->grav[1] = enabled && c->grid.num_dim > 1 ? gy : 0.0;
    c->grav[2] = enabled && c->grid.num_dim > 2 ? gz : 0.0;
    return MC_OK;
}

mc_status mc_slab_unique_id(uint8_t* id) {
    if (!id) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null id");
    }
    const char* why = "";
    if (!mc::slab_unique_id(id, &why)) {
        return fail(MC_ERR_UNSUPPORTED, std::string("mc_slab_unique_id: ") + why);
    }
    return MC_OK;
}

mc_status mc_set_slab_decomposition(mc_ctx* c, const uint8_t* id, int32_t rank, int32_t world) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!id || world < 1 || rank < 0 || rank >= world) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null id or rank outside [0, world)");
    }
    if (c->grid.num_dim < 2) {
        return fail(MC_ERR_UNSUPPORTED, "slab decomposition splits y (2D) or z (3D)");
    }
    if (c->slab) {
        return fail(MC_ERR_INVALID_ARGUMENT, "the context already holds a slab decomposition");
    }
    const int axis = c->grid.num_dim - 1;
    const int f0 = 2 * axis;
    if ((c->grid.bc[f0] == MC_BC_PERIODIC) != (c->grid.bc[f0 + 1] == MC_BC_PERIODIC)) {
        return fail(MC_ERR_INVALID_ARGUMENT, "periodic boundaries come in pairs");
    }
    const bool periodic = c->grid.bc[f0] == MC_BC_PERIODIC;
    const int n = axis == 1 ? c->ny : c->nz;
    const char* why = "";
    mc::SlabExchange* s = mc::slab_create(id, rank, world, axis, n, c->grid.ng, c->grid.xc, c->grid.yc,
                                          c->grid.zc, c->nvar, periodic, &why);
    if (!s) {
        return fail(MC_ERR_CUDA, std::string("slab communicator: ") + why);
    }
    c->slab = s;
    c->slab_faces = mc::slab_face_mask(s);
    if (c->grid.num_dim == 2) {
        if (mc_status st = create_overlap(c)) {
            return st;
        }
    }
    // the kernels leave the exchanged faces' ghosts alone
    for (int f = f0; f < f0 + 2; ++f) {
        if ((c->slab_faces >> f) & 1) {
            c->grid.bc[f] = MC_BC_USERFN;
        }
    }
    return MC_OK;
}

mc_status mc_set_cfl_reduce_hook(mc_ctx* c, void (*fn)(void*, uint64_t*, void*), void* user) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    c->cfl_hook = fn;
    c->cfl_hook_data = user;
    return MC_OK;
}

mc_status mc_set_eos(mc_ctx* c, int32_t type, double avg_mass, int32_t include_ionisation_energy,
                     const mc_eos_table* t) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (type < MC_EOS_IDEAL || type > MC_EOS_TABULATED_LTE_H || !(avg_mass > 0.0)) {
        return fail(MC_ERR_INVALID_ARGUMENT, "unknown EOS type or avg_mass <= 0");
    }
    if (type == MC_EOS_TABULATED_LTE_H &&
        (!t || !t->y_table || !t->log_T_table || t->n_eint_rho < 1 || t->n_rho < 1 ||
         !(t->log_eint_rho_step > 0.0) || !(t->log_rho_step > 0.0))) {
        return fail(MC_ERR_INVALID_ARGUMENT, "the tabulated EOS needs a table with positive steps");
    }
    c->eos_type = type;
    c->eos_avg_mass = avg_mass;
    c->eos_ion = include_ionisation_energy ? 1 : 0;
    if (type == MC_EOS_IDEAL) {
        return MC_OK;
    }
    const size_t cells = (size_t)c->plane;
    if (!c->eos_y) {
        MC_CUDA(cudaMalloc(&c->eos_y, sizeof(double) * cells), "EOS fields");
        MC_CUDA(cudaMalloc(&c->eos_T, sizeof(double) * cells), "EOS fields");
    }
    // Eos::init_* (source/Eos.cpp:40-86): the tabulated kind starts from
    // y_space = -1, which makes its first energy shift zero
    std::vector<double> init(cells, type == MC_EOS_TABULATED_LTE_H ? -1.0 : 0.0);
    MC_CUDA(cudaMemcpy(c->eos_y, init.data(), sizeof(double) * cells, cudaMemcpyHostToDevice), "EOS fields");
    MC_CUDA(cudaMemset(c->eos_T, 0, sizeof(double) * cells), "EOS fields");
    if (type == MC_EOS_TABULATED_LTE_H) {
        const size_t n = (size_t)t->n_rho * (size_t)t->n_eint_rho;
        cudaFree(c->eos_ytab);
        cudaFree(c->eos_lTtab);
        c->eos_ytab = c->eos_lTtab = nullptr;
        MC_CUDA(cudaMalloc(&c->eos_ytab, sizeof(double) * n), "EOS table");
        MC_CUDA(cudaMalloc(&c->eos_lTtab, sizeof(double) * n), "EOS table");
        MC_CUDA(cudaMemcpy(c->eos_ytab, t->y_table, sizeof(double) * n, cudaMemcpyHostToDevice), "EOS table");
        MC_CUDA(cudaMemcpy(c->eos_lTtab, t->log_T_table, sizeof(double) * n, cudaMemcpyHostToDevice), "EOS table");
        c->tab_x0 = t->log_eint_rho_start;
        c->tab_dx = t->log_eint_rho_step;
        c->tab_nx = t->n_eint_rho;
        c->tab_y0 = t->log_rho_start;
        c->tab_dy = t->log_rho_step;
        c->tab_ny = t->n_rho;
        if (!c->buf_eos) {
            MC_CUDA(cudaMalloc(&c->buf_eos, c->state_bytes), "EOS stage buffer");
        }
    }
    return MC_OK;
}

mc_status mc_update_eos(mc_ctx* c, double* Q, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!Q) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null Q");
    }
    if (c->eos_type == MC_EOS_IDEAL) {
        return MC_OK;
    }
    c->launches += 1;
    MC_CUDA(mc::launch_eos_update(eos_launch(c, Q, Q, false), c->grid.num_dim, (cudaStream_t)stream), "EOS update");
    return MC_OK;
}

mc_status mc_get_eos_fields(mc_ctx* c, double* y, double* T, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (c->eos_type == MC_EOS_IDEAL || !c->eos_y) {
        return fail(MC_ERR_INVALID_ARGUMENT, "no non-ideal EOS selected");
    }
    const size_t bytes = sizeof(double) * (size_t)c->plane;
    const cudaStream_t s = (cudaStream_t)stream;
    if (y) {
        MC_CUDA(cudaMemcpyAsync(y, c->eos_y, bytes, cudaMemcpyDefault, s), "EOS fields");
    }
    if (T) {
        MC_CUDA(cudaMemcpyAsync(T, c->eos_T, bytes, cudaMemcpyDefault, s), "EOS fields");
    }
    return MC_OK;
}

mc_status mc_get_prim(mc_ctx* c, const double* Q, double* W, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    const double* src = c->last_stage_in ? c->last_stage_in : Q;
    if (!W || !src) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null W, or null Q before the first step");
    }
    StageParams p = base_params(c);
    p.q_in = src;
    c->launches += 1;
    MC_CUDA(mc::launch_cons_to_prim(p, W, c->grid.num_dim, (cudaStream_t)stream), "cons_to_prim launch");
    return MC_OK;
}

mc_status mc_fill_bcs(mc_ctx* c, double* Q, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!Q) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null Q");
    }
    StageParams p = base_params(c);
    p.q_in = Q;
    p.q_out = Q;
    c->launches += 1;
    MC_CUDA(mc::launch_fill_bcs(p, c->grid.num_dim, (cudaStream_t)stream), "fill_bcs");
    if (mc_status st = exchange_slab(c, Q, (cudaStream_t)stream)) {
        return st;
    }
    if (c->user_bc) {
        c->user_bc(c->user_bc_data, Q, stream);
    }
    return MC_OK;
}

mc_status mc_compute_dt(mc_ctx* c, const double* Q, const mc_clock* clock, double* dt_out, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!Q || !dt_out) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    StageParams p = base_params(c);
    p.q_in = Q;
    c->launches += 2;
    MC_CUDA(mc::launch_cfl_min(p, c->grid.num_dim, s), "cfl_min");
    if (mc_status st = reduce_cfl(c, s)) {
        return st;
    }
    MC_CUDA(cudaMemcpyAsync(c->blk_host, c->blk, sizeof(mc::DeviceBlock), cudaMemcpyDeviceToHost, s), "read-back");
    MC_CUDA(cudaStreamSynchronize(s), "sync");
    double m;
    std::memcpy(&m, &c->blk_host->cfl_min_bits, sizeof(double));
    double dt = m * c->scheme.max_cfl;
    if (clock) {
        dt = clamp_to_output(dt, clock);
    }
    *dt_out = dt;
    return MC_OK;
}

mc_status mc_time_step(mc_ctx* c, double* Q, double dt, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!Q) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null Q");
    }
    if (!(dt > 0.0) || !std::isfinite(dt)) {
        return fail(MC_ERR_INVALID_ARGUMENT, "dt must be positive and finite");
    }
    if (mc_status st = check_user_bc(c)) {
        return st;
    }
    c->min_from_clock = false;
    return enqueue_step(c, Q, dt, nullptr, true, (cudaStream_t)stream);
}

mc_status mc_advance(mc_ctx* c, double* Q, mc_clock* clock, int64_t max_steps, int64_t* steps_done,
                     double* dt_log, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!Q || !clock || max_steps < 0) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null Q / clock or negative max_steps");
    }
    if (mc_status st = check_user_bc(c)) {
        return st;
    }
    const cudaStream_t s = (cudaStream_t)stream;
    if (dt_log && c->dt_log_cap < max_steps + 1) {
        cudaFree(c->dt_log);
        c->dt_log = nullptr;
        c->dt_log_cap = 0;
        MC_CUDA(cudaMalloc(&c->dt_log, sizeof(double) * (size_t)(max_steps + 1)), "dt log");
        c->dt_log_cap = max_steps + 1;
    }
    double* dlog = dt_log ? c->dt_log : nullptr;
    c->min_from_clock = true;
    MC_CUDA(mc::launch_clock_init(c->blk, clock->time, clock->max_time, clock->prev_output_time,
                                  clock->output_delta, c->scheme.max_cfl, s),
            "clock init");
    StageParams p = base_params(c);
    p.q_in = Q;
    MC_CUDA(mc::launch_cfl_min(p, c->grid.num_dim, s), "cfl_min");
    if (mc_status st = reduce_cfl(c, s)) {
        return st;
    }
    MC_CUDA(mc::launch_clock_advance(c->blk, dlog, 1, s), "clock");
    c->launches += 4;
    const double* dt_dev = &c->blk->dt;
    const int64_t chunk = 64;
    int64_t issued = 0;
    while (issued < max_steps) {
        const int64_t n = std::min(chunk, max_steps - issued);
        for (int64_t k = 0; k < n; ++k) {
            if (mc_status st = enqueue_step(c, Q, 0.0, dt_dev, false, s)) {
                return st;
            }
            if (mc_status st = reduce_cfl(c, s)) {
                return st;
            }
            MC_CUDA(mc::launch_clock_advance(c->blk, dlog, 0, s), "clock");
            c->launches += 1;
        }
        issued += n;
        if (issued < max_steps) {
            MC_CUDA(cudaMemcpyAsync(c->blk_host, c->blk, sizeof(mc::DeviceBlock), cudaMemcpyDeviceToHost, s),
                    "read-back");
            MC_CUDA(cudaStreamSynchronize(s), "sync");
            if (c->blk_host->done) {
                break;
            }
        }
    }
    MC_CUDA(cudaMemcpyAsync(c->blk_host, c->blk, sizeof(mc::DeviceBlock), cudaMemcpyDeviceToHost, s), "read-back");
    MC_CUDA(cudaStreamSynchronize(s), "sync");
    const mc::DeviceBlock& b = *c->blk_host;
    clock->time = b.time;
    clock->prev_output_time = b.prev_output_time;
    if (steps_done) {
        *steps_done = b.steps;
    }
    if (dt_log && b.steps > 0) {
        MC_CUDA(cudaMemcpy(dt_log, c->dt_log, sizeof(double) * (size_t)b.steps, cudaMemcpyDeviceToHost),
                "dt log read-back");
    }
    return MC_OK;
}

mc_status mc_last_cfl_min(mc_ctx* c, double* cfl_min, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!cfl_min) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    MC_CUDA(cudaMemcpyAsync(c->blk_host, c->blk, sizeof(mc::DeviceBlock), cudaMemcpyDeviceToHost, s), "read-back");
    MC_CUDA(cudaStreamSynchronize(s), "sync");
    if (c->min_from_clock) {
        *cfl_min = c->blk_host->last_cfl_min;
    } else {
        std::memcpy(cfl_min, &c->blk_host->cfl_min_bits, sizeof(double));
    }
    return MC_OK;
}

mc_status mc_get_status(mc_ctx* c, uint32_t* flags, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!flags) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    const cudaStream_t s = (cudaStream_t)stream;
    MC_CUDA(cudaMemcpyAsync(c->blk_host, c->blk, sizeof(mc::DeviceBlock), cudaMemcpyDeviceToHost, s), "read-back");
    MC_CUDA(cudaStreamSynchronize(s), "sync");
    *flags = c->blk_host->status;
    const unsigned zero = 0;
    MC_CUDA(cudaMemcpyAsync(&c->blk->status, &zero, sizeof(unsigned), cudaMemcpyHostToDevice, s), "clear");
    MC_CUDA(cudaStreamSynchronize(s), "sync");
    return MC_OK;
}

mc_status mc_step_host(mc_ctx* c, double* Q_host, double* Q, const mc_clock* clock, double* dt_out, void* stream) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!Q_host || !Q || !dt_out) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    if (mc_status st = check_user_bc(c)) {
        return st;
    }
    const cudaStream_t s = (cudaStream_t)stream;
    if (host_pipelined(c)) {
        return step_host_pipelined(c, Q_host, Q, clock, dt_out, s);
    }
    MC_CUDA(cudaMemcpyAsync(Q, Q_host, c->state_bytes, cudaMemcpyHostToDevice, s), "state in");
    double dt = 0.0;
    if (mc_status st = mc_compute_dt(c, Q, clock, &dt, stream)) {
        return st;
    }
    *dt_out = dt;
    if (mc_status st = mc_time_step(c, Q, dt, stream)) {
        return st;
    }
    MC_CUDA(cudaMemcpyAsync(Q_host, Q, c->state_bytes, cudaMemcpyDeviceToHost, s), "state out");
    MC_CUDA(cudaStreamSynchronize(s), "sync");
    return MC_OK;
}

mc_status mc_set_slab_overlap(mc_ctx* c, int32_t enable) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    c->slab_overlap = enable != 0;
    return MC_OK;
}

mc_status mc_profile_stages(mc_ctx* c, int32_t enable) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    for (auto& t : c->timed) {
        c->event_pool.push_back(t.start);
        c->event_pool.push_back(t.stop);
        if (t.start2) {
            c->event_pool.push_back(t.start2);
            c->event_pool.push_back(t.stop2);
        }
    }
    c->timed.clear();
    c->profiling = enable != 0;
    return MC_OK;
}

mc_status mc_stage_time(mc_ctx* c, int32_t kind, double* total_ms, int64_t* launches) {
    if (mc_status st = check_ctx(c)) {
        return st;
    }
    if (!total_ms || !launches) {
        return fail(MC_ERR_INVALID_ARGUMENT, "null argument");
    }
    double sum = 0.0;
    int64_t n = 0;
    for (auto& t : c->timed) {
        if (t.kind != kind) {
            continue;
        }
        MC_CUDA(cudaEventSynchronize(t.stop), "event sync");
        float ms = 0.0f;
        MC_CUDA(cudaEventElapsedTime(&ms, t.start, t.stop), "event time");
        if (t.start2) {
            // the two pieces of an overlapped stage: first start to last stop
            MC_CUDA(cudaEventSynchronize(t.stop2), "event sync");
            float s2 = 0.0f, e2 = 0.0f;
            MC_CUDA(cudaEventElapsedTime(&s2, t.start, t.start2), "event time");
            MC_CUDA(cudaEventElapsedTime(&e2, t.start, t.stop2), "event time");
            ms = std::max(ms, e2) - std::min(0.0f, s2);
        }
        sum += ms;
        ++n;
    }
    *total_ms = sum;
    *launches = n;
    return MC_OK;
}

int64_t mc_launch_count(const mc_ctx* c) {
    return c ? c->launches : 0;
}

} // extern "C"
