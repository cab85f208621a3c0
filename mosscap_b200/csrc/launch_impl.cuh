// Launchers of the stage kernels for one dimension (MC_DIM) and one compute
// type (MC_REAL). Each stage_d<dim>_<precision>.cu translation unit defines
// the two macros and includes this file, so the template instantiations of
// the different dimensions and precisions compile in parallel.
#pragma once

#include <cuda_runtime.h>

#include <cstring>

#include "launch.h"
#include "stage_kernels.cuh"

#ifndef MC_DIM
#error "MC_DIM must be defined"
#endif
#ifndef MC_REAL
#error "MC_REAL must be defined"
#endif
#ifndef MC_LAUNCH_NAME
#error "MC_LAUNCH_NAME must be defined"
#endif
// MC_SRC 1: the variants with a registered source term (mc_set_gravity);
// they compile in their own translation units.
#ifndef MC_SRC
#define MC_SRC 0
#endif
// MC_DEFER 1 (2D): the deferred form of the stage kernel, whose tiles write
// only their x+y divergence (for mc_step_host); in units of their own, so
// the regular kernels compile as before.
#ifndef MC_DEFER
#define MC_DEFER 0
#endif

namespace mc {
namespace {

using Real = MC_REAL;

inline int cdiv(long long a, long long b) {
    return (int)((a + b - 1) / b);
}

// Raise the dynamic shared-memory limit of a kernel once per process.
template <class K>
cudaError_t allow_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) {
        return cudaSuccess;
    }
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// The TMA tile load applies when the kernel has a TMA form for this
// reconstruction and still fits its CTAs per SM, the tile's x start is even
// (ng - H even), there are no tracers, and the stage input's tensor map can
// be built (16-byte aligned base, even row length, box inside the array).
template <int NDIM, int REC>
bool use_tma(const StageParams& p, CUtensorMap* map) {
    using G = TileGeom<2, REC>;
    if (!tma_capable<NDIM, REC, Real>(p.nvar) || p.ntracer != 0 || ((p.ng - G::H) & 1) != 0) {
        return false;
    }
    std::memset(map, 0, sizeof(*map));
    return tma_map_for(p.q_in, p.xc, p.yc, p.zc, p.nvar, G::WX, G::WY, 2 + NDIM, map);
}

// The tiled kernel (2D stage, or the 3D x-y plane pass) with or without the
// TMA tile load.
template <int NDIM, int REC, int LIM, int RS, bool SRC, bool TMA>
cudaError_t launch_tiled(const StageParams& p, const CUtensorMap& map, cudaStream_t s) {
    if constexpr (TMA && !tma_capable<NDIM, REC, Real>(2 + NDIM)) {
        return cudaErrorNotSupported;  // never taken: use_tma refused it
    } else {
        auto k = stage2d_kernel<NDIM, REC, LIM, RS, Real, SRC, TMA, (NDIM == 2 && MC_DEFER != 0)>;
        const size_t sm = TMA ? smem_bytes_tma<NDIM, REC, Real>(p.nvar) : smem_bytes<NDIM, REC, Real>(p.nvar);
        cudaError_t e = allow_smem(k, sm);
        if (e != cudaSuccess) {
            return e;
        }
        const int rows = (NDIM == 2 && p.tile_rows > 0) ? p.tile_rows : cdiv(p.ny, kTile);
        const dim3 grid(cdiv(p.nx, kTile), rows, NDIM == 3 ? p.nz : 1);
        k<<<grid, dim3(tile_threads<NDIM, Real>()), sm, s>>>(p, map);
        return cudaGetLastError();
    }
}

// The z pass with a TMA tile load where the staging area fits its CTAs per
// SM, there are no tracers and the state's tensor map can be built.
template <int REC>
bool use_ztile_tma(const StageParams& p, CUtensorMap* map) {
    if (!ztile_tma_capable<REC, Real>() || p.ntracer != 0) {
        return false;
    }
    return tma_map_for(p.q_in, p.xc, p.yc, p.zc, p.nvar, kZStageX, 1, 5, map, ZTileGeom<REC>::WZ);
}

template <int REC, int LIM, int RS, bool TMA>
cudaError_t launch_ztile(const StageParams& p, const CUtensorMap& map, cudaStream_t s) {
    if constexpr (TMA && !ztile_tma_capable<REC, Real>()) {
        return cudaErrorNotSupported;  // never taken: use_ztile_tma refused it
    } else {
        auto k = ztile3d_kernel<REC, LIM, RS, Real, MC_SRC, TMA>;
        const size_t sm = TMA ? ztile_smem_bytes_tma<REC, Real>() : ztile_smem_bytes<REC, Real>(p.nvar);
        cudaError_t e = allow_smem(k, sm);
        if (e != cudaSuccess) {
            return e;
        }
        k<<<dim3(cdiv(p.nz, kTile), cdiv(p.nx, kZCols), p.ny), dim3(kThreads), sm, s>>>(p, map);
        return cudaGetLastError();
    }
}

template <int REC, int LIM, int RS>
cudaError_t launch_one(const StageParams& p, int pass, cudaStream_t s) {
#if MC_DIM == 1
    (void)pass;
    auto k = stage1d_kernel<REC, LIM, RS, Real, MC_SRC>;
    const size_t sm = smem_bytes<1, REC, Real>(p.nvar);
    cudaError_t e = allow_smem(k, sm);
    if (e != cudaSuccess) {
        return e;
    }
    k<<<dim3(cdiv(p.nx, kWarps * kTile)), dim3(kThreads), sm, s>>>(p);
#elif MC_DIM == 2
    (void)pass;
    CUtensorMap map;
    if (use_tma<2, REC>(p, &map)) {
        return launch_tiled<2, REC, LIM, RS, MC_SRC, true>(p, map, s);
    }
    return launch_tiled<2, REC, LIM, RS, MC_SRC, false>(p, map, s);
#else
    if (pass == 0) {
        CUtensorMap map;
        const cudaError_t e = use_tma<3, REC>(p, &map) ? launch_tiled<3, REC, LIM, RS, false, true>(p, map, s)
                                                      : launch_tiled<3, REC, LIM, RS, false, false>(p, map, s);
        if (e != cudaSuccess) {
            return e;
        }
    } else {
        CUtensorMap map;
        std::memset(&map, 0, sizeof(map));
        const cudaError_t e = use_ztile_tma<REC>(p, &map) ? launch_ztile<REC, LIM, RS, true>(p, map, s)
                                                          : launch_ztile<REC, LIM, RS, false>(p, map, s);
        if (e != cudaSuccess) {
            return e;
        }
    }
#endif
    return cudaGetLastError();
}

template <int REC, int LIM>
cudaError_t by_solver(const StageParams& p, int rs, int pass, cudaStream_t s) {
    switch (rs) {
        case kRusanov:
            return launch_one<REC, LIM, kRusanov>(p, pass, s);
        case kHll:
            return launch_one<REC, LIM, kHll>(p, pass, s);
        default:
            return launch_one<REC, LIM, kHllc>(p, pass, s);
    }
}

} // namespace

// Dispatch on (reconstruction, limiter, solver). The limiter only matters for
// MUSCL and PPM; FOG and WENO5-Z are limiter-agnostic (Reconstruct.hpp:33-44).
// In 2D, pass 2 is the finishing of a stage whose tiles wrote only their
// divergence (finish2d_kernel), whatever the scheme.
cudaError_t MC_LAUNCH_NAME(const StageParams& p, int rec, int lim, int rs, int pass, cudaStream_t s) {
#if MC_DIM == 2 && !MC_DEFER
    if (pass == 2) {
        const long long cells = (long long)p.nx * p.ny;
        const long long want = (cells + kThreads - 1) / kThreads;
        const int blocks = (int)(want < 148LL * 8 ? want : 148LL * 8);
        finish2d_kernel<Real, MC_SRC><<<blocks, kThreads, 0, s>>>(p);
        return cudaGetLastError();
    }
#endif
    switch (rec) {
        case kFog:
            return by_solver<kFog, kMonotonizedCentral>(p, rs, pass, s);
        case kMuscl:
            switch (lim) {
                case kVanLeer:
                    return by_solver<kMuscl, kVanLeer>(p, rs, pass, s);
                case kMonotonizedCentral:
                    return by_solver<kMuscl, kMonotonizedCentral>(p, rs, pass, s);
                default:
                    return by_solver<kMuscl, kMinmod>(p, rs, pass, s);
            }
        case kPpm:
            switch (lim) {
                case kVanLeer:
                    return by_solver<kPpm, kVanLeer>(p, rs, pass, s);
                case kMonotonizedCentral:
                    return by_solver<kPpm, kMonotonizedCentral>(p, rs, pass, s);
                default:
                    return by_solver<kPpm, kMinmod>(p, rs, pass, s);
            }
        default:
            return by_solver<kWeno5z, kMonotonizedCentral>(p, rs, pass, s);
    }
}

} // namespace mc
