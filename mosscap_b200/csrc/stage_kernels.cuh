// Fused SSPRK stage kernels.
//
// One launch performs one stage of the reference's time_step
// (source/TimeStepping.cpp) for a whole grid:
//   global_cons_to_prim -> reconstruct / Riemann flux per axis ->
//   integrate_flux + stage combination -> fill_bcs
// (source/Hydro.cpp:8-166, source/TimeStepping.cpp:10-35, Boundaries.hpp)
// without any intermediate array in global memory: the primitive tile, the
// face states and the fluxes live in shared memory and registers.
//
// Work decomposition (1D / 2D, and the x-y part of 3D):
//   * a CTA owns a tile of TX x TY output cells (TX = TY = 30 in 2D);
//   * phase 1 loads the tile plus a cross-shaped halo of H cells, converts
//     to primitives once per cell and stores them in shared memory;
//   * a y sweep gives one warp per column: lane L reconstructs cell L-1
//     (cells -1..30), receives the left state of its face from lane L-1 with
//     a shuffle, solves the Riemann problem for the face below its cell, and
//     takes the next face's flux from lane L+1 -- every face is solved once
//     and every cell is reconstructed once per axis; the y divergence goes to
//     shared memory;
//   * an x sweep does the same with one warp per row, and the lane of each
//     cell then combines both divergences with the stage inputs, writes the
//     new state, scatters the ghost cells it is the source of, and (last
//     stage) reduces the CFL minimum and status flags.
// 3D splits each stage in two launches: the x-y plane pass above writes the
// x+y divergence per cell, then a z pass (tiles of x columns by z cells,
// one warp-wide sweep per column) adds the z divergence and finishes the
// stage.
#pragma once

#include "common.cuh"
#include "tma.cuh"

namespace mc {

constexpr int kThreads = 256; // threads per CTA of the 1D and z-pass kernels (2D: tile_threads)
constexpr int kWarps = kThreads / 32;
// CTAs per SM of the 256-thread kernels: FP64 three (80 registers a
// thread), FP32 four (64 registers; measured faster than three despite a
// few spills).
constexpr int kMinBlocks2d = 3;
constexpr int kMinBlocks2dF32 = 4;

// Shared-memory geometry of the tiled kernels.
template <int NDIM, int REC>
struct TileGeom {
    static constexpr int H = halo_of<REC>();
    static constexpr int TX = kTile;
    static constexpr int TY = NDIM == 1 ? 1 : kTile;
    static constexpr int WX = TX + 2 * H;                    // stored columns
    static constexpr int P = (WX % 2 == 0) ? WX + 1 : WX;    // odd pitch: conflict-free columns
    static constexpr int WY = NDIM == 1 ? 1 : TY + 2 * H;    // stored rows
    static constexpr int PY = TX + 1;                        // odd pitch of the y divergence
};

// Element counts of the per-variable shared arrays (1D uses a different
// layout: NW segments of TX cells).
template <int NDIM, int REC>
__host__ __device__ constexpr int smem_w_per_var() {
    using G = TileGeom<NDIM, REC>;
    return NDIM == 1 ? kWarps * (kTile + 2 * G::H) : G::WY * G::P;
}
template <int NDIM, int REC>
__host__ __device__ constexpr int smem_dqy_per_var() {
    using G = TileGeom<NDIM, REC>;
    return NDIM == 1 ? 0 : G::TY * G::PY;
}
template <int NDIM, int REC, class T>
__host__ __device__ constexpr size_t smem_bytes(int nvar) {
    return sizeof(T) * (size_t)nvar * (smem_w_per_var<NDIM, REC>() + smem_dqy_per_var<NDIM, REC>());
}

// Shared memory of the tiled kernels with a TMA tile load: a 128-byte
// aligned region that first holds the conserved tile as the TMA copies it
// (WY rows x WX cells x 2 + NDIM variables, doubles; corners included) and
// later the y divergences (it is free once the tile is converted), then the
// primitive tile W.
template <int NDIM, int REC>
__host__ __device__ constexpr size_t tma_stage_bytes() {
    using G = TileGeom<2, REC>;
    return sizeof(double) * (size_t)(2 + NDIM) * G::WY * G::WX;
}
template <int NDIM, int REC, class T>
__host__ __device__ constexpr size_t tma_region_bytes(int nvar) {
    const size_t dy = sizeof(T) * (size_t)nvar * smem_dqy_per_var<2, REC>();
    const size_t st = tma_stage_bytes<NDIM, REC>();
    return ((dy > st ? dy : st) + 127) / 128 * 128;
}
template <int NDIM, int REC, class T>
__host__ __device__ constexpr size_t smem_bytes_tma(int nvar) {
    return 128 + tma_region_bytes<NDIM, REC, T>(nvar) + sizeof(T) * (size_t)nvar * smem_w_per_var<2, REC>();
}

__device__ __forceinline__ long long qidx(const StageParams& p, int v, int k, int j, int i) {
    return (((long long)v * p.zc + k) * p.yc + j) * (long long)p.xc + i;
}

// CFL time-step bound and status flags of one written conserved state.
// FP64 path (T = double): the reference's dt_reducer (source/Hydro.cpp:
// 192-206) from cons_to_prim, bit for bit. FP32 form (T = float): the same
// bound in FP64 arithmetic from 1 / rho formed once (two FP64 divisions
// instead of five in 3D): p = (gamma - 1)(E - |m|^2 / 2 rho),
// c_s = sqrt(gamma p / rho), |v| = |m| / rho.
template <int NDIM, class T>
__device__ __forceinline__ double cfl_bound_of(const StageParams& p, const double* q, unsigned* flags) {
    constexpr int nh = 2 + NDIM;
    bool fin = true;
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        fin = fin && isfinite(q[v]);
    }
    if constexpr (sizeof(T) == 8) {
        double w[nh];
        prim_from_cons<NDIM>(p.gamma, q, w);
        *flags |= state_flags(w[0], w[nh - 1], fin);
        return cfl_dt<NDIM>(p.gamma, p.dx, w);
    } else {
        const double inv = 1.0 / q[0];
        double m2 = q[1] * q[1];
        if constexpr (NDIM > 1) {
            m2 += q[2] * q[2];
        }
        if constexpr (NDIM > 2) {
            m2 += q[3] * q[3];
        }
        const double pr = (p.gamma - 1.0) * (q[1 + NDIM] - 0.5 * m2 * inv);
        *flags |= state_flags(q[0], pr, fin);
        const double cs = sqrt(p.gamma * pr * inv);
        return p.dx / (cs + sqrt(m2) * inv);
    }
}

// Write the new value of interior cell (i, j, k); returns its CFL bound
// (last stage) and ORs its status flags into *flags.
template <int NDIM, class T = double>
__device__ __forceinline__ double write_own(const StageParams& p, int i, int j, int k, const double* qn,
                                            bool want_dt, unsigned* flags) {
    const long long vs = (long long)p.zc * p.yc * p.xc;  // variable stride of the state
    double* dst = p.q_out + qidx(p, 0, k, j, i);
#pragma unroll
    for (int v = 0; v < kMaxVars; ++v) {
        if (v < p.nvar) {
            dst[v * vs] = qn[v];
        }
    }
    return want_dt ? cfl_bound_of<NDIM, T>(p, qn, flags) : __longlong_as_double(0x7ff0000000000000ll);
}

// Write every ghost that interior cell (i, j, k), of new value qn, is the
// source of; returns the CFL minimum over the written ghosts (last stage) and
// ORs their status flags into *flags. The ghost targets along each axis are
// enumerated one at a time (axis_target_at), so nothing goes to local memory.
template <int NDIM, class T = double>
__device__ __forceinline__ double scatter_ghosts(const StageParams& p, int i, int j, int k, const double* qn,
                                                 bool want_dt, unsigned* flags) {
    const int nvar = p.nvar;
    double dtmin = __longlong_as_double(0x7ff0000000000000ll);
    auto account = [&](const double* q) {
        if (want_dt) {
            dtmin = smin(cfl_bound_of<NDIM, T>(p, q, flags), dtmin);
        }
    };
    const long long vs = (long long)p.zc * p.yc * p.xc;  // variable stride of the state
    const bool nx_ = near_face(i, p.nx, p.ng);
    const bool ny_ = NDIM > 1 && near_face(j, p.ny, p.ng);
    const bool nz_ = NDIM > 2 && near_face(k, p.nz, p.ng);
    if (!(nx_ || ny_ || nz_)) {
        return dtmin;
    }
    const int sx = start_target_count(i, p.nx, p.ng, p.bc.kind[0]);
    const int cx = 1 + sx + end_target_count(i, p.nx, p.ng, p.bc.kind[1]);
    int sy = 0, cy = 1, sz = 0, cz = 1;
    if constexpr (NDIM > 1) {
        sy = start_target_count(j, p.ny, p.ng, p.bc.kind[2]);
        cy = 1 + sy + end_target_count(j, p.ny, p.ng, p.bc.kind[3]);
    }
    if constexpr (NDIM > 2) {
        sz = start_target_count(k, p.nz, p.ng, p.bc.kind[4]);
        cz = 1 + sz + end_target_count(k, p.nz, p.ng, p.bc.kind[5]);
    }
    // each ghost target starts again from the cell's new state and applies
    // the face transforms of its axes in x, y, z order, as the sequential
    // per-axis fill does; only two states are live at a time
    for (int a = 0; a < cx; ++a) {
        int fa;
        const int ia = axis_target_at(i, p.nx, p.ng, p.bc.kind[0], p.bc.kind[1], sx, a, &fa);
        for (int b = 0; b < cy; ++b) {
            int fb = -1;
            const int jb = NDIM > 1 ? axis_target_at(j, p.ny, p.ng, p.bc.kind[2], p.bc.kind[3], sy, b, &fb) : j;
            for (int c = 0; c < cz; ++c) {
                if (a == 0 && b == 0 && c == 0) {
                    continue;
                }
                int fc = -1;
                const int kc = NDIM > 2 ? axis_target_at(k, p.nz, p.ng, p.bc.kind[4], p.bc.kind[5], sz, c, &fc) : k;
                double qc[kMaxVars];
#pragma unroll
                for (int v = 0; v < kMaxVars; ++v) {
                    qc[v] = qn[v];
                }
                if (fa >= 0) {
                    bc_transform<NDIM>(p.bc, 0, fa, nvar, qc);
                }
                if (fb >= 0) {
                    bc_transform<NDIM>(p.bc, 1, fb, nvar, qc);
                }
                if (fc >= 0) {
                    bc_transform<NDIM>(p.bc, 2, fc, nvar, qc);
                }
                double* dst = p.q_out + qidx(p, 0, kc, jb, ia);
#pragma unroll
                for (int v = 0; v < kMaxVars; ++v) {
                    if (v < nvar) {
                        dst[v * vs] = qc[v];
                    }
                }
                account(qc);
            }
        }
    }
    return dtmin;
}

// Every ghost cell of a 1D or 2D state, from the stored new values of the
// interior cells next to a face: the cells whose scatter_ghosts has
// targets, shared out over `count` threads starting at `first`. The values
// are read through L2 (they were written by other CTAs, which fenced their
// stores before the caller learned they were done). Returns the CFL minimum
// over the ghosts (last stage) and ORs their flags into *flags: with each
// cell's own store (write_own), the same values and bounds as write_cell.
template <int NDIM, class T>
__device__ double fill_ghosts(const StageParams& p, int first, int count, unsigned* flags) {
    const int ng = p.ng, nx = p.nx, ny = NDIM > 1 ? p.ny : 1;
    const long long vs = (long long)p.zc * p.yc * p.xc;
    const int xc_near = nx < 2 * ng ? nx : 2 * ng;                  // interior columns next to an x face
    const int yr_near = NDIM > 1 ? (ny < 2 * ng ? ny : 2 * ng) : 1; // interior rows next to a y face (1D: the one row)
    const long long n_near_rows = NDIM > 1 ? (long long)yr_near * nx : 0;
    const long long n_far = (long long)(ny - (NDIM > 1 ? yr_near : 0)) * xc_near;
    double dtmin = __longlong_as_double(0x7ff0000000000000ll);
    for (long long t = first; t < n_near_rows + n_far; t += count) {
        int ii, jj;
        if (t < n_near_rows) {
            const int r = (int)(t / nx);
            ii = (int)(t - (long long)r * nx);
            jj = (r < ng || yr_near < 2 * ng) ? r : ny - yr_near + r;
        } else {
            const long long u = t - n_near_rows;
            const int q = (int)(u / xc_near);
            const int cc = (int)(u - (long long)q * xc_near);
            jj = NDIM > 1 ? ng + q : 0;
            ii = (cc < ng || xc_near < 2 * ng) ? cc : nx - xc_near + cc;
        }
        const int i = ng + ii;
        const int j = NDIM > 1 ? ng + jj : 0;
        const double* src = p.q_out + qidx(p, 0, 0, j, i);
        double qn[kMaxVars];
#pragma unroll
        for (int v = 0; v < kMaxVars; ++v) {
            qn[v] = v < p.nvar ? __ldcg(src + v * vs) : 0.0;
        }
        dtmin = smin(scatter_ghosts<NDIM, T>(p, i, j, 0, qn, p.last != 0, flags), dtmin);
    }
    return dtmin;
}

// Write the new value of interior cell (i, j, k) and every ghost it is the
// source of; returns the CFL minimum over the written values (last stage) and
// ORs their status flags into *flags.
template <int NDIM, class T = double>
__device__ __forceinline__ double write_cell(const StageParams& p, int i, int j, int k, double* qn,
                                             bool want_dt, unsigned* flags) {
    const double own = write_own<NDIM, T>(p, i, j, k, qn, want_dt, flags);
    return smin(scatter_ghosts<NDIM, T>(p, i, j, k, qn, want_dt, flags), own);
}

// Primitives of a cell for the sweep of compute type T. T = double: the
// reference's cons_to_prim (Eos.hpp:61-79), bit for bit. T = float (the FP32
// compute form, whose sweep rounds to FP32 anyway): 1 / rho is formed once
// in FP64, the velocities are m / rho through it, and the pressure is
// recovered in FP64 from the total energy with the kinetic energy
// |m|^2 / (2 rho), so that the cancellation E - e_kin of high-Mach and
// near-vacuum cells stays an FP64 operation -- one FP64 division per cell
// instead of 2 + (NDIM > 1) + (NDIM > 2).
template <int NDIM, class T>
__device__ __forceinline__ void prim_for_sweep(double gamma, const double* q, double* w) {
    if constexpr (sizeof(T) == 8) {
        prim_from_cons<NDIM>(gamma, q, w);
    } else {
        const double inv = 1.0 / q[0];
        double m2 = q[1] * q[1];
        w[0] = q[0];
        w[1] = q[1] * inv;
        if constexpr (NDIM > 1) {
            m2 += q[2] * q[2];
            w[2] = q[2] * inv;
        }
        if constexpr (NDIM > 2) {
            m2 += q[3] * q[3];
            w[3] = q[3] * inv;
        }
        w[1 + NDIM] = (gamma - 1.0) * (q[1 + NDIM] - 0.5 * m2 * inv);
    }
}

// Load one cell's conserved variables from q_in and store its primitives
// (tracers divided by rho, source/Hydro.cpp:27-33) into shared memory.
template <int NDIM, class T>
__device__ __forceinline__ unsigned load_prim(const StageParams& p, int k, int j, int i, bool inb, T* w_smem,
                                              int var_stride) {
    constexpr int nh = 2 + NDIM;
    double q[nh], w[nh];
    const long long vs = (long long)p.zc * p.yc * p.xc;  // variable stride of the state
    const long long id0 = qidx(p, 0, k, j, i);
    if (inb) {
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            q[v] = p.q_in[id0 + v * vs];
        }
    } else {
        // outside the array: a benign state that no stored result depends on
        q[0] = 1.0;
#pragma unroll
        for (int v = 1; v < nh - 1; ++v) {
            q[v] = 0.0;
        }
        q[nh - 1] = 1.0;
    }
    prim_for_sweep<NDIM, T>(p.gamma, q, w);
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        w_smem[v * var_stride] = T(w[v]);
    }
    if (p.ntracer > 0) {
        const double inv_rho = 1.0 / q[0];
        for (int t = 0; t < p.ntracer; ++t) {
            const double qt = inb ? p.q_in[id0 + (nh + t) * vs] : 0.0;
            w_smem[(nh + t) * var_stride] = T(qt * inv_rho);
        }
    }
    if (!inb) {
        return 0u;
    }
    bool fin = true;
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        fin = fin && isfinite(q[v]);
    }
    return state_flags(w[0], w[nh - 1], fin);
}

// The same as load_prim for a cell whose conserved variables sit in the
// TMA-staged tile (variable stride stg_vs doubles); no tracers.
template <int NDIM, class T>
__device__ __forceinline__ unsigned staged_prim(const StageParams& p, const double* src, int stg_vs, bool inb,
                                                T* w_smem, int var_stride) {
    constexpr int nh = 2 + NDIM;
    double q[nh], w[nh];
    if (inb) {
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            q[v] = src[v * stg_vs];
        }
    } else {
        // outside the array: a benign state that no stored result depends on
        q[0] = 1.0;
#pragma unroll
        for (int v = 1; v < nh - 1; ++v) {
            q[v] = 0.0;
        }
        q[nh - 1] = 1.0;
    }
    prim_for_sweep<NDIM, T>(p.gamma, q, w);
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        w_smem[v * var_stride] = T(w[v]);
    }
    if (!inb) {
        return 0u;
    }
    bool fin = true;
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        fin = fin && isfinite(q[v]);
    }
    return state_flags(w[0], w[nh - 1], fin);
}

// Variables reconstructed per iteration of the sweep's variable loop. The
// 2D WENO5-Z sweep is instruction-fetch bound when its four
// reconstructions are unrolled (instruction-cache hit rate 63 %); two per
// iteration measured 5 % faster on KH 2048^2 than four, and one per
// iteration 3 %; with 320-thread CTAs and 96 registers the unrolled form
// is still 0.6 % slower. Everything else is fully unrolled (one PPM
// reconstruction per iteration made the 3D plane pass 4 % slower).
template <int NDIM, int REC>
__host__ __device__ constexpr int recon_group() {
    return (REC == kWeno5z && NDIM == 2) ? 2 : 2 + NDIM;
}

// One warp-wide face sweep along `axis` (warp-uniform): lane L reconstructs
// the cell whose stencil centre is `centre` (cell L-1 of the segment), solves
// the face on its left, and returns in d[] the divergence F(left) - F(right)
// of its cell (meaningful on lanes 1..kTile). `stride` is the distance between
// neighbouring cells along the axis in shared memory, `vstride` between
// variables. The axis is a runtime value so that both directions run the
// same instructions.
template <int NDIM, int REC, int LIM, int RS, class T>
__device__ __forceinline__ void face_sweep(const T* centre, int stride, int vstride, int ntracer, T gamma, T gfac,
                                           int axis, T* d, T* d_tr) {
    constexpr int nh = 2 + NDIM;
    constexpr int S = stencil_half<REC>();
    constexpr int G = recon_group<NDIM, REC>();
    T wl[nh], wr[nh];
    if constexpr (G < nh) {
        // a rolled loop over groups of G variables (a smaller instruction
        // footprint); the results rotate through wl / wr so that they stay
        // in registers and end in variable order
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            wl[v] = T(0);
            wr[v] = T(0);
        }
#pragma unroll 1
        for (int v0 = 0; v0 < nh; v0 += G) {
            T a[G], b[G];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                T s[5];
#pragma unroll
                for (int o = -S; o <= S; ++o) {
                    s[2 + o] = centre[(v0 + g) * vstride + o * stride];
                }
                reconstruct<REC, LIM>(s, a[g], b[g]);
            }
#pragma unroll
            for (int u = 0; u < nh - G; ++u) {
                wl[u] = wl[u + G];
                wr[u] = wr[u + G];
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                wl[nh - G + g] = a[g];
                wr[nh - G + g] = b[g];
            }
        }
    } else {
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            T s[5];
#pragma unroll
            for (int o = -S; o <= S; ++o) {
                s[2 + o] = centre[v * vstride + o * stride];
            }
            reconstruct<REC, LIM>(s, wl[v], wr[v]);
        }
    }
    T left[nh];
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        left[v] = __shfl_up_sync(0xffffffffu, wr[v], 1);
    }
    T f[nh];
    riemann<RS, NDIM>(gamma, gfac, axis, left, wl, f);
#pragma unroll
    for (int v = 0; v < nh; ++v) {
        const T fn = __shfl_down_sync(0xffffffffu, f[v], 1);
        d[v] = f[v] - fn;
    }
    // passive tracers: upwinded by the sign of the mass flux (Hydro.cpp:155-162)
    for (int t = 0; t < ntracer; ++t) {
        T s[5];
#pragma unroll
        for (int o = -S; o <= S; ++o) {
            s[2 + o] = centre[(nh + t) * vstride + o * stride];
        }
        T tl, tr;
        reconstruct<REC, LIM>(s, tl, tr);
        const T tleft = __shfl_up_sync(0xffffffffu, tr, 1);
        const T ft = (f[0] >= T(0)) ? f[0] * tleft : f[0] * tl;
        const T fn = __shfl_down_sync(0xffffffffu, ft, 1);
        d_tr[t] = ft - fn;
    }
}

// ---------------------------------------------------------------------------
// 1D: one warp updates one segment of kTile cells, independently of the
// other warps of its CTA (so one CTA can serve segments of different
// problems in a batch). W is this warp's shared window of
// nvar x (kTile + 2H) primitives.
// ---------------------------------------------------------------------------
template <int REC>
__host__ __device__ constexpr int seg1d_window() {
    return kTile + 2 * halo_of<REC>();
}

// SCATTER false: only the cell itself is stored (the batched kernel fills a
// problem's ghosts once all its cells are written: fill_ghosts).
template <int REC, int LIM, int RS, class T, bool SRC = false, bool SCATTER = true>
__device__ __forceinline__ void segment1d(const StageParams& p, int x0, T* W, double& dtmin, unsigned& flags) {
    constexpr int NDIM = 1;
    constexpr int nh = 3;
    constexpr int H = halo_of<REC>();
    constexpr int WN = seg1d_window<REC>();
    const int lane = threadIdx.x & 31;
    for (int it = lane; it < WN; it += 32) {
        const int i = p.ng + x0 - H + it;  // array index
        const bool inb = i >= 0 && i < p.xc;
        flags |= load_prim<NDIM, T>(p, 0, 0, i, inb, W + it, WN);
    }
    __syncwarp();
    const int cl = lane - 1;  // cell of this lane, relative to x0
    T d[nh], d_tr[kMaxVars];
    const T gfac = T((p.gamma + 1.0) / (2.0 * p.gamma));
    face_sweep<NDIM, REC, LIM, RS, T>(W + H + cl, 1, WN, p.ntracer, T(p.gamma), gfac, 0, d, d_tr);
    __syncwarp();  // the window may be reloaded by the caller's next segment

    const double dt = stage_dt(p);
    const double dtdx = dt / p.dx;
    const int cell = x0 + cl;  // interior index
    if (lane >= 1 && lane <= kTile && cell < p.nx) {
        const int i = cell + p.ng;
        double qn[kMaxVars];
#pragma unroll
        for (int v = 0; v < kMaxVars; ++v) {
            qn[v] = 0.0;
        }
        const bool old = combo_reads_old(p.combo);
        double sdt[nh];
        source_dt<1, SRC>(p, 0, 0, i, dt, sdt);
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            double qu = 0.0;
            qu += double(d[v]);
            qu *= dtdx;
            const long long id = qidx(p, v, 0, 0, i);
            qn[v] = combine(p.combo, old ? p.q_old[id] : 0.0, p.q_in[id], qu, sdt[v]);
        }
        // constant tracer slots keep qn in registers
#pragma unroll
        for (int t = 0; t < kMaxVars - nh; ++t) {
            if (t < p.ntracer) {
                double qu = 0.0;
                qu += double(d_tr[t]);
                qu *= dtdx;
                const long long id = qidx(p, nh + t, 0, 0, i);
                qn[nh + t] = combine(p.combo, old ? p.q_old[id] : 0.0, p.q_in[id], qu, 0.0);
            }
        }
        if constexpr (SCATTER) {
            dtmin = smin(write_cell<NDIM, T>(p, i, 0, 0, qn, p.last != 0, &flags), dtmin);
        } else {
            dtmin = smin(write_own<NDIM, T>(p, i, 0, 0, qn, p.last != 0, &flags), dtmin);
        }
    }
}

// 1D stage kernel: warp w of CTA b updates segment b * kWarps + w.
template <int REC, int LIM, int RS, class T, bool SRC = false>
__global__ void __launch_bounds__(kThreads) stage1d_kernel(StageParams p) {
    if (p.dt_dev && p.blk->done) {
        return;
    }
    maybe_reset_min(p);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_d[kWarps];
    __shared__ unsigned red_u[kWarps];
    const int warp = threadIdx.x >> 5;
    T* W = reinterpret_cast<T*>(smem_raw) + (size_t)warp * p.nvar * seg1d_window<REC>();
    double dtmin = __longlong_as_double(0x7ff0000000000000ll);
    unsigned flags = 0;
    const int x0 = (blockIdx.x * kWarps + warp) * kTile;
    if (x0 < p.nx) {
        segment1d<REC, LIM, RS, T, SRC>(p, x0, W, dtmin, flags);
    }
    block_publish(dtmin, flags, p.last != 0, p.blk, red_d, red_u);
}

// ---------------------------------------------------------------------------
// 2D stage kernel, and the x-y pass of 3D (NDIM == 3: one z plane per
// blockIdx.z, writing the x+y divergence instead of finishing the stage).
// ---------------------------------------------------------------------------
// One CTA updates tile (bx, by) of a 2D problem, or of z plane bz in the 3D
// plane pass. smem holds nvar x (WY x P) primitives and nvar x (TY x PY)
// y divergences. Contains CTA-wide barriers: every thread of the CTA calls it.
//
// TMA: smem is a 128-byte aligned region laid out as smem_bytes_tma
// describes; the conserved tile arrives by one tensor copy (tmap, completed
// on mbar) instead of per-thread loads. Without TMA, smem holds W and then
// the y divergences (smem_bytes).
template <int NDIM, int REC, int LIM, int RS, class T, bool SRC = false, int NT = kThreads, bool TMA = false,
          bool DEFER = false, bool SCATTER = true>
__device__ __forceinline__ void tile2d(const StageParams& p, int bx, int by, int bz, T* smem, double& dtmin,
                                       unsigned& flags, const CUtensorMap* tmap = nullptr, uint64_t* mbar = nullptr) {
    constexpr int nh = 2 + NDIM;
    constexpr int NW = NT / 32;
    using G = TileGeom<2, REC>;
    constexpr int H = G::H, TX = G::TX, TY = G::TY, WX = G::WX, P = G::P, WY = G::WY, PY = G::PY;
    constexpr int WV = WY * P;   // per-variable stride of W
    constexpr int YV = TY * PY;  // per-variable stride of dFy
    T* W;
    T* DY;
    if constexpr (TMA) {
        DY = smem;
        W = reinterpret_cast<T*>(reinterpret_cast<unsigned char*>(smem) + tma_region_bytes<NDIM, REC, T>(p.nvar));
    } else {
        W = smem;
        DY = W + (size_t)p.nvar * WV;
    }

    const int x0 = bx * TX;
    const int y0 = by * TY;
    const int k = NDIM == 3 ? p.ng + bz : 0;
    const int vw = min(TX, p.nx - x0);
    const int vh = min(TY, p.ny - y0);

    // phase 1: primitives of the tile and its cross-shaped halo
    constexpr int core = TY * WX;
    constexpr int items = core + 2 * H * TX;
    if constexpr (TMA) {
        // the box of WX x WY cells around the tile (x start even: the host
        // only takes this path when ng - H is even), all hydro variables;
        // cells outside the array arrive as zeros and are replaced below
        double* stg = reinterpret_cast<double*>(smem);
        if (threadIdx.x == 0) {
            mbar_init(mbar, 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            mbar_expect_tx(mbar, (uint32_t)tma_stage_bytes<NDIM, REC>());
            if constexpr (NDIM == 3) {
                tma_load_4d(stg, tmap, p.ng + x0 - H, p.ng + y0 - H, k, 0, mbar);
            } else {
                tma_load_3d(stg, tmap, p.ng + x0 - H, p.ng + y0 - H, 0, mbar);
            }
        }
        const bool ok = mbar_wait_bounded(mbar, 0, kTmaWaitPolls);
        if (!__syncthreads_and(ok)) {
            // the copy did not complete: raise the flag, give the copy in
            // flight one more bounded wait, and leave the tile unwritten
            if (threadIdx.x == 0) {
                atomicOr(&p.blk->status, 0x20u);
            }
            mbar_wait_bounded(mbar, 0, kTmaWaitPolls);
            __syncthreads();
            return;
        }
        for (int it = threadIdx.x; it < items; it += NT) {
            int tx, ty;
            if (it < core) {
                ty = it / WX;
                tx = it - ty * WX - H;
            } else {
                const int r = it - core;
                const int hr = r / TX;
                tx = r - hr * TX;
                ty = hr < H ? hr - H : TY + hr - H;
            }
            const int i = p.ng + x0 + tx;
            const int j = p.ng + y0 + ty;
            const bool inb = i >= 0 && i < p.xc && j >= 0 && j < p.yc;
            flags |= staged_prim<NDIM, T>(p, stg + (ty + H) * WX + (tx + H), WX * WY, inb,
                                          W + (ty + H) * P + (tx + H), WV);
        }
    } else {
        for (int it = threadIdx.x; it < items; it += NT) {
            int tx, ty;
            if (it < core) {
                ty = it / WX;
                tx = it - ty * WX - H;
            } else {
                const int r = it - core;
                const int hr = r / TX;
                tx = r - hr * TX;
                ty = hr < H ? hr - H : TY + hr - H;
            }
            const int i = p.ng + x0 + tx;
            const int j = p.ng + y0 + ty;
            const bool inb = i >= 0 && i < p.xc && j >= 0 && j < p.yc;
            flags |= load_prim<NDIM, T>(p, k, j, i, inb, W + (ty + H) * P + (tx + H), WV);
        }
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const T gamma = T(p.gamma);
    const T gfac = T((p.gamma + 1.0) / (2.0 * p.gamma));
    const int ntr = p.ntracer;
    const double dt = stage_dt(p);
    const double dtdx = dt / p.dx;
    const bool old = combo_reads_old(p.combo);
    const int c = lane - 1;  // this lane's cell along the sweep

    // Two passes through one copy of the sweep code. Pass 0: y faces, one warp
    // per column, divergence into DY. Pass 1: x faces, one warp per row; the
    // lane of each cell then finishes it: q_update = (0 + dFx) + dFy as in
    // integrate_flux (source/TimeStepping.cpp:22-27), the stage combination,
    // the store and the ghost scatter (2D), or the x+y divergence (3D).
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        const int axis = 1 - pass;
        const int nlines = axis == 1 ? vw : vh;
        for (int line = warp; line < nlines; line += NW) {
            const T* centre = axis == 0 ? W + (line + H) * P + (c + H) : W + (c + H) * P + (line + H);
            T d[nh], d_tr[kMaxVars];
            face_sweep<NDIM, REC, LIM, RS, T>(centre, axis == 0 ? 1 : P, WV, ntr, gamma, gfac, axis, d, d_tr);
            const bool mine = lane >= 1 && lane <= kTile;
            if (axis == 1) {
                if (mine) {
                    T* dst = DY + c * PY + line;
#pragma unroll
                    for (int v = 0; v < nh; ++v) {
                        dst[v * YV] = d[v];
                    }
                    for (int t = 0; t < ntr; ++t) {
                        dst[(nh + t) * YV] = d_tr[t];
                    }
                }
                continue;
            }
            if (!mine || c >= vw) {
                continue;
            }
            const T* dfy = DY + line * PY + c;
            const int i = p.ng + x0 + c;
            const int j = p.ng + y0 + line;
            // 3D, and the deferred form of a 2D stage (finished later by
            // finish2d_kernel once dt is known): the x+y divergence only
            if constexpr (NDIM == 3 || DEFER) {
                const long long cells = (long long)p.nx * p.ny * p.nz;
                const long long kz = NDIM == 3 ? k - p.ng : 0;
                const long long o = (kz * p.ny + (j - p.ng)) * p.nx + (i - p.ng);
#pragma unroll
                for (int v = 0; v < nh; ++v) {
                    double qu = 0.0;
                    qu += double(d[v]);
                    qu += double(dfy[v * YV]);
                    p.dqxy[v * cells + o] = qu;
                }
                for (int t = 0; t < ntr; ++t) {
                    double qu = 0.0;
                    qu += double(d_tr[t]);
                    qu += double(dfy[(nh + t) * YV]);
                    p.dqxy[(nh + t) * cells + o] = qu;
                }
            } else {
                double qn[kMaxVars];
#pragma unroll
                for (int v = 0; v < kMaxVars; ++v) {
                    qn[v] = 0.0;
                }
                const long long vs = (long long)p.zc * p.yc * p.xc;  // variable stride of the state
                const long long id0 = qidx(p, 0, 0, j, i);
                double qo[nh], qi[nh], qu[nh], sdt[nh];
#pragma unroll
                for (int v = 0; v < nh; ++v) {
                    qi[v] = p.q_in[id0 + v * vs];
                    qo[v] = old ? p.q_old[id0 + v * vs] : 0.0;
                }
                source_dt_of<NDIM, SRC>(p, qi, dt, sdt);
#pragma unroll
                for (int v = 0; v < nh; ++v) {
                    qu[v] = 0.0;
                    qu[v] += double(d[v]);
                    qu[v] += double(dfy[v * YV]);
                    qu[v] *= dtdx;
                }
                combine_all<nh>(p.combo, qo, qi, qu, sdt, qn);
                // constant tracer slots keep qn in registers (a loop up to
                // ntr would index it at run time and put it in local memory)
#pragma unroll
                for (int t = 0; t < kMaxVars - nh; ++t) {
                    if (t < ntr) {
                        double qt = 0.0;
                        qt += double(d_tr[t]);
                        qt += double(dfy[(nh + t) * YV]);
                        qt *= dtdx;
                        const long long id = id0 + (nh + t) * vs;
                        qn[nh + t] = combine(p.combo, old ? p.q_old[id] : 0.0, p.q_in[id], qt, 0.0);
                    }
                }
                if constexpr (SCATTER) {
                    dtmin = smin(write_cell<NDIM, T>(p, i, j, 0, qn, p.last != 0, &flags), dtmin);
                } else {
                    dtmin = smin(write_own<NDIM, T>(p, i, j, 0, qn, p.last != 0, &flags), dtmin);
                }
            }
        }
        __syncthreads();
    }
}

// The rest of a 2D stage whose tiles wrote only their x+y divergence
// (p.dqxy, [var][y][x] over the interior cells): per interior cell, x
// fastest, q_update = that divergence times dt / dx, the source term, the
// stage combination, the store and the ghost scatter, as the tile's own
// finishing does with the same operations in the same order. Lets a step
// compute stage 0's fluxes before dt is known.
template <class T, bool SRC>
__global__ void __launch_bounds__(kThreads) finish2d_kernel(StageParams p) {
    if (p.dt_dev && p.blk->done) {
        return;
    }
    constexpr int NDIM = 2;
    constexpr int nh = 4;
    __shared__ double red_d[kWarps];
    __shared__ unsigned red_u[kWarps];
    double dtmin = __longlong_as_double(0x7ff0000000000000ll);
    unsigned flags = 0;
    const double dt = stage_dt(p);
    const double dtdx = dt / p.dx;
    const bool old = combo_reads_old(p.combo);
    const int ntr = p.ntracer;
    const long long cells = (long long)p.nx * p.ny;
    const long long vs = (long long)p.zc * p.yc * p.xc;
    for (long long o = blockIdx.x * (long long)kThreads + threadIdx.x; o < cells;
         o += (long long)gridDim.x * kThreads) {
        const int y = (int)(o / p.nx);
        const int x = (int)(o - (long long)y * p.nx);
        const int i = p.ng + x, j = p.ng + y;
        const long long id0 = qidx(p, 0, 0, j, i);
        double qo[nh], qi[nh], qu[nh], sdt[nh];
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            qi[v] = p.q_in[id0 + v * vs];
            qo[v] = old ? p.q_old[id0 + v * vs] : 0.0;
        }
        source_dt_of<NDIM, SRC>(p, qi, dt, sdt);
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            qu[v] = p.dqxy[v * cells + o];
            qu[v] *= dtdx;
        }
        double qn[kMaxVars];
#pragma unroll
        for (int v = nh; v < kMaxVars; ++v) {
            qn[v] = 0.0;
        }
        combine_all<nh>(p.combo, qo, qi, qu, sdt, qn);
#pragma unroll
        for (int t = 0; t < kMaxVars - nh; ++t) {
            if (t < ntr) {
                double qt = p.dqxy[(nh + t) * cells + o];
                qt *= dtdx;
                const long long id = id0 + (nh + t) * vs;
                qn[nh + t] = combine(p.combo, old ? p.q_old[id] : 0.0, p.q_in[id], qt, 0.0);
            }
        }
        dtmin = smin(write_cell<NDIM, T>(p, i, j, 0, qn, p.last != 0, &flags), dtmin);
    }
    block_publish(dtmin, flags, p.last != 0, p.blk, red_d, red_u);
}

// Threads per CTA of the tiled stage kernel and CTAs per SM it is compiled
// for. A sweep pass has 30 lines: with 10 warps every warp takes exactly
// three (with 8, six warps take four and two take three).
//   2D FP64: two CTAs of 320 threads per SM (20 warps, up to 96 registers,
//     72 KB of shared memory each): 3 % faster on KH 2048^2 than three CTAs
//     of 256 at 80 registers, 24 % faster in the batched form.
//   2D FP32: three CTAs of 320 threads (64 registers, a few spilled): 3 %
//     faster than four of 256.
//   3D FP64 plane pass: five variables' tiles take 90 KB of shared memory,
//     two CTAs per SM; 384 threads (24 warps at 80 registers) measured 2 %
//     faster than 320 and 11 % faster than 256.
template <int NDIM, class T>
__host__ __device__ constexpr int tile_threads() {
    return NDIM == 1 ? kThreads : ((NDIM == 3 && sizeof(T) == 8) ? 384 : 320);
}
template <int NDIM, class T>
__host__ __device__ constexpr int tile_min_blocks() {
    return NDIM == 1 ? (sizeof(T) == 4 ? kMinBlocks2dF32 : kMinBlocks2d) : (sizeof(T) == 4 ? 3 : 2);
}

// Whether the TMA tile load fits the kernel's CTAs per SM (shared memory
// of one SM: 228 KB, 1 KB of it reserved per CTA) and its halo allows an
// even x start with the usual ng (MUSCL's two-cell halo does not with ng = 3).
template <int NDIM, int REC, class T>
__host__ __device__ constexpr bool tma_capable(int nvar) {
    return REC != kMuscl &&
           (size_t)tile_min_blocks<NDIM, T>() * (smem_bytes_tma<NDIM, REC, T>(nvar) + 1024 + 256) <= 233472;
}

// DEFER (2D): the tiles write only their x+y divergence into p.dqxy.
template <int NDIM, int REC, int LIM, int RS, class T, bool SRC = false, bool TMA = false, bool DEFER = false>
__global__ void __launch_bounds__(tile_threads<NDIM, T>(), tile_min_blocks<NDIM, T>())
    stage2d_kernel(StageParams p, const __grid_constant__ CUtensorMap tmap) {
    if (p.dt_dev && p.blk->done) {
        return;
    }
    maybe_reset_min(p);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NT = tile_threads<NDIM, T>();
    __shared__ double red_d[NT / 32];
    __shared__ unsigned red_u[NT / 32];
    __shared__ __align__(8) uint64_t mbar;
    double dtmin = __longlong_as_double(0x7ff0000000000000ll);
    unsigned flags = 0;
    unsigned char* base = smem_raw;
    if constexpr (TMA) {
        // the tensor copy's destination: 128-byte aligned
        base += (128u - (smem_addr(smem_raw) & 127u)) & 127u;
    }
    const int by = (int)blockIdx.y + ((int)blockIdx.y >= p.row_split ? p.row_skip : 0);
    // 2D WENO5-Z in FP64: the finishing pass stores only the tile's own
    // cells; the ghosts whose sources lie in the tile (edge tiles only)
    // follow in a second loop, so the scatter's divergence and registers
    // stay out of the finishing pass (KH 2048^2 stage 0.603 -> 0.597 ms).
    // The other forms keep the scatter in the finishing pass: with the
    // second loop the FP32 form's spills grew from 232 to 640 bytes of
    // stores, and the FP64 FOG, MUSCL and PPM kernels with HLLC went from
    // none to about 490.
    constexpr bool kAfter = NDIM == 2 && !DEFER && sizeof(T) == 8 && REC == kWeno5z;
    tile2d<NDIM, REC, LIM, RS, T, SRC, NT, TMA, DEFER, !kAfter>(p, blockIdx.x, by, blockIdx.z,
                                                                reinterpret_cast<T*>(base), dtmin, flags, &tmap, &mbar);
    if constexpr (kAfter) {
        const int x0 = blockIdx.x * kTile, y0 = by * kTile;
        const int vw = min(kTile, p.nx - x0), vh = min(kTile, p.ny - y0);
        if (x0 < p.ng || x0 + vw > p.nx - p.ng || y0 < p.ng || y0 + vh > p.ny - p.ng) {
            __syncthreads();
            const long long vs = (long long)p.zc * p.yc * p.xc;
            for (int it = threadIdx.x; it < vw * vh; it += NT) {
                const int ty = it / vw, tx = it - ty * vw;
                const int i = p.ng + x0 + tx, j = p.ng + y0 + ty;
                if (!(near_face(i, p.nx, p.ng) || near_face(j, p.ny, p.ng))) {
                    continue;
                }
                // the cell's new state as this CTA stored it
                const double* src = p.q_out + qidx(p, 0, 0, j, i);
                double qn[kMaxVars];
#pragma unroll
                for (int v = 0; v < kMaxVars; ++v) {
                    qn[v] = v < p.nvar ? __ldcg(src + v * vs) : 0.0;
                }
                dtmin = smin(scatter_ghosts<NDIM, T>(p, i, j, 0, qn, p.last != 0, &flags), dtmin);
            }
        }
    }
    block_publish(dtmin, flags, NDIM != 3 && p.last != 0, p.blk, red_d, red_u);
}

// ---------------------------------------------------------------------------
// 3D z pass: adds the z divergence to the x+y divergence from the plane
// pass and finishes the stage (passive tracers included).
// ---------------------------------------------------------------------------
// Tile of the z pass: kZCols x-columns (one coalesced 256-byte row per
// variable) by kTile z cells of one y row, with H halo rows above and below.
constexpr int kZCols = 32;

template <int REC>
struct ZTileGeom {
    static constexpr int H = halo_of<REC>();
    static constexpr int TZ = kTile;
    static constexpr int WZ = TZ + 2 * H;  // stored rows (z)
    static constexpr int PZ = kZCols + 1;  // odd pitch: conflict-free z columns
    static constexpr int WV = WZ * PZ;     // per-variable stride
};

template <int REC, class T>
__host__ __device__ constexpr size_t ztile_smem_bytes(int nvar) {
    return sizeof(T) * (size_t)nvar * ZTileGeom<REC>::WV;
}

// The z pass with a TMA tile load: the conserved tile (kZStageX x-columns
// from the even column at or before the tile's first, one y row, WZ z rows,
// five variables, doubles) is staged by one tensor copy ahead of the
// primitive tile W; it stays there for the finishing phase, which takes each
// cell's stage input from it. 128 bytes of slack align the staging area.
constexpr int kZStageX = kZCols + 2;
template <int REC>
__host__ __device__ constexpr size_t ztile_stage_bytes() {
    return sizeof(double) * 5 * (size_t)ZTileGeom<REC>::WZ * kZStageX;
}
template <int REC, class T>
__host__ __device__ constexpr size_t ztile_smem_bytes_tma() {
    return 128 + ztile_stage_bytes<REC>() + ztile_smem_bytes<REC, T>(5);
}
// CTAs per SM of the z pass: three (80 registers); the TMA form only where
// its staging area still lets three fit (the FP32 form: 72.8 KB per CTA).
template <int REC, class T>
__host__ __device__ constexpr bool ztile_tma_capable() {
    return (size_t)kMinBlocks2d * (ztile_smem_bytes_tma<REC, T>() + 1024 + 256) <= 233472;
}

// z pass: each CTA loads the primitives of its tile, sweeps every column
// along z with one warp (lane L reconstructs cell L-1 of the column, solves
// the face below it, and takes the next face's flux from lane L+1, exactly
// like the x-y sweeps), overwrites the column with its z divergence -- no
// other warp reads that column -- and then finishes each cell in row order
// (coalesced): q_update = dq_xy + dFz as the x, y, z flux sum of
// integrate_flux (source/TimeStepping.cpp:22-27), the stage combination, the
// store and the ghost scatter. Grid: (z chunks, x tiles, y rows), z chunks
// fastest, so the halo rows a neighbouring chunk re-reads are still in L2.
// Three CTAs per SM in both precisions: at four (64 registers) the FP32 z
// pass spilled 196 bytes per thread.
//
// TMA (no tracers, even row length; see ztile_tma_capable): the conserved
// tile arrives by one tensor copy (tmap: 4D x, y, z, var; box kZStageX x 1 x
// WZ x 5) completed on an mbarrier with a bounded wait, and the finishing
// phase reads each cell's stage input from it.
template <int REC, int LIM, int RS, class T, bool SRC = false, bool TMA = false>
__global__ void __launch_bounds__(kThreads, kMinBlocks2d)
    ztile3d_kernel(StageParams p, const __grid_constant__ CUtensorMap tmap) {
    if (p.dt_dev && p.blk->done) {
        return;
    }
    maybe_reset_min(p);
    constexpr int NDIM = 3;
    constexpr int nh = 5;
    using G = ZTileGeom<REC>;
    constexpr int H = G::H, TZ = G::TZ, WZ = G::WZ, PZ = G::PZ, WV = G::WV;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ double red_d[kWarps];
    __shared__ unsigned red_u[kWarps];
    __shared__ __align__(8) uint64_t mbar;
    T* W;
    double* stg = nullptr;
    if constexpr (TMA) {
        unsigned char* base = smem_raw + ((128u - (smem_addr(smem_raw) & 127u)) & 127u);
        stg = reinterpret_cast<double*>(base);
        W = reinterpret_cast<T*>(base + ztile_stage_bytes<REC>());
    } else {
        W = reinterpret_cast<T*>(smem_raw);
    }

    const int z0 = blockIdx.x * TZ;
    const int x0 = blockIdx.y * kZCols;
    const int yi = blockIdx.z;
    const int j = p.ng + yi;
    const int vw = min(kZCols, p.nx - x0);
    const int vh = min(TZ, p.nz - z0);
    unsigned flags = 0;
    double dtmin = __longlong_as_double(0x7ff0000000000000ll);

    // phase 1: primitives of the tile and its halo rows
    // (TMA: column x of the tile is column x + xoff of the staged box)
    const int xoff = (p.ng + x0) & 1;
    if constexpr (TMA) {
        if (threadIdx.x == 0) {
            mbar_init(&mbar, 1);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            mbar_expect_tx(&mbar, (uint32_t)ztile_stage_bytes<REC>());
            tma_load_4d(stg, &tmap, p.ng + x0 - xoff, j, p.ng + z0 - H, 0, &mbar);
        }
        const bool ok = mbar_wait_bounded(&mbar, 0, kTmaWaitPolls);
        if (!__syncthreads_and(ok)) {
            // the copy did not complete: raise the flag, give the copy in
            // flight one more bounded wait, and leave the tile unwritten
            if (threadIdx.x == 0) {
                atomicOr(&p.blk->status, 0x20u);
            }
            mbar_wait_bounded(&mbar, 0, kTmaWaitPolls);
            __syncthreads();
            return;
        }
        constexpr int SV = WZ * kZStageX;  // per-variable stride of the staged box
        for (int it = threadIdx.x; it < WZ * kZCols; it += kThreads) {
            const int r = it / kZCols;
            const int x = it - r * kZCols;
            const int k = p.ng + z0 - H + r;
            const bool inb = x < vw && k >= 0 && k < p.zc;
            flags |= staged_prim<NDIM, T>(p, stg + r * kZStageX + x + xoff, SV, inb, W + r * PZ + x, WV);
        }
    } else {
        for (int it = threadIdx.x; it < WZ * kZCols; it += kThreads) {
            const int r = it / kZCols;
            const int x = it - r * kZCols;
            const int i = p.ng + x0 + x;
            const int k = p.ng + z0 - H + r;
            const bool inb = x < vw && k >= 0 && k < p.zc;
            flags |= load_prim<NDIM, T>(p, k, j, i, inb, W + r * PZ + x, WV);
        }
    }
    __syncthreads();

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const T gamma = T(p.gamma);
    const T gfac = T((p.gamma + 1.0) / (2.0 * p.gamma));
    const int ntr = p.ntracer;
    const int c = lane - 1;  // this lane's cell along the column

    // phase 2: z sweeps, one warp per column; the divergence replaces the
    // column's primitives once every lane has read its stencil
#pragma unroll 1
    for (int col = warp; col < vw; col += kWarps) {
        T* centre = W + (c + H) * PZ + col;
        T d[nh], d_tr[kMaxVars];
        face_sweep<NDIM, REC, LIM, RS, T>(centre, PZ, WV, ntr, gamma, gfac, 2, d, d_tr);
        __syncwarp();
        if (lane >= 1 && lane <= TZ) {
#pragma unroll
            for (int v = 0; v < nh; ++v) {
                centre[v * WV] = d[v];
            }
            for (int t = 0; t < ntr; ++t) {
                centre[(nh + t) * WV] = d_tr[t];
            }
        }
    }
    __syncthreads();

    // phase 3: finish every cell of the tile, x fastest
    const double dt = stage_dt(p);
    const double dtdx = dt / p.dx;
    const bool old = combo_reads_old(p.combo);
    const long long cells = (long long)p.nx * p.ny * p.nz;
    const long long vs = (long long)p.zc * p.yc * p.xc;  // variable stride of the state
#pragma unroll 1
    for (int it = threadIdx.x; it < TZ * kZCols; it += kThreads) {
        const int zr = it / kZCols;
        const int x = it - zr * kZCols;
        if (x >= vw || zr >= vh) {
            continue;
        }
        const int i = p.ng + x0 + x;
        const int kk = p.ng + z0 + zr;
        const long long o = ((long long)(z0 + zr) * p.ny + yi) * p.nx + (x0 + x);
        const long long id0 = qidx(p, 0, kk, j, i);
        const T* dz = W + (zr + H) * PZ + x;
        double qo[nh], qi[nh], qu[nh], sdt[nh];
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            qu[v] = p.dqxy[v * cells + o];
            if constexpr (TMA) {
                qi[v] = stg[(v * WZ + zr + H) * kZStageX + x + xoff];
            } else {
                qi[v] = p.q_in[id0 + v * vs];
            }
            qo[v] = old ? p.q_old[id0 + v * vs] : 0.0;
        }
        source_dt_of<NDIM, SRC>(p, qi, dt, sdt);
#pragma unroll
        for (int v = 0; v < nh; ++v) {
            qu[v] += double(dz[v * WV]);
            qu[v] *= dtdx;
        }
        double qn[kMaxVars];
#pragma unroll
        for (int v = nh; v < kMaxVars; ++v) {
            qn[v] = 0.0;
        }
        combine_all<nh>(p.combo, qo, qi, qu, sdt, qn);
        // constant tracer slots keep qn in registers
#pragma unroll
        for (int t = 0; t < kMaxVars - nh; ++t) {
            if (t < ntr) {
                double qt = p.dqxy[(nh + t) * cells + o];
                qt += double(dz[(nh + t) * WV]);
                qt *= dtdx;
                const long long id = id0 + (nh + t) * vs;
                qn[nh + t] = combine(p.combo, old ? p.q_old[id] : 0.0, p.q_in[id], qt, 0.0);
            }
        }
        dtmin = smin(write_own<NDIM, T>(p, i, j, kk, qn, p.last != 0, &flags), dtmin);
    }
    // the ghost scatter as a second loop, only in tiles with a cell next to
    // a face: its registers stay out of the finishing loop above
    const bool near_tile = (p.ng + x0 < 2 * p.ng) || (p.ng + x0 + vw - 1 >= p.nx) || near_face(j, p.ny, p.ng) ||
                           (p.ng + z0 < 2 * p.ng) || (p.ng + z0 + vh - 1 >= p.nz);
    if (near_tile) {
#pragma unroll 1
        for (int it = threadIdx.x; it < TZ * kZCols; it += kThreads) {
            const int zr = it / kZCols;
            const int x = it - zr * kZCols;
            const int i = p.ng + x0 + x;
            const int kk = p.ng + z0 + zr;
            if (x >= vw || zr >= vh || !(near_face(i, p.nx, p.ng) || near_face(j, p.ny, p.ng) ||
                                         near_face(kk, p.nz, p.ng))) {
                continue;
            }
            // this thread's own store of the cell, read back
            const long long id0 = qidx(p, 0, kk, j, i);
            double qn[kMaxVars];
#pragma unroll
            for (int v = 0; v < kMaxVars; ++v) {
                qn[v] = v < p.nvar ? p.q_out[id0 + v * vs] : 0.0;
            }
            dtmin = smin(scatter_ghosts<NDIM, T>(p, i, j, kk, qn, p.last != 0, &flags), dtmin);
        }
    }
    block_publish(dtmin, flags, p.last != 0, p.blk, red_d, red_u);
}

} // namespace mc
