// Host side of the TMA tile loads (tma.cuh): tensor maps of state arrays.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstring>
#include <mutex>

#include "tma.cuh"

namespace mc {

namespace {

PFN_cuTensorMapEncodeTiled encode_fn() {
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
        }
    });
    return fn;
}

struct Entry {
    const double* q;
    int xc, yc, zc, nvar, bx, by, nv, bz;
    CUtensorMap map;
};

constexpr int kCache = 16;
Entry g_cache[kCache];
int g_used = 0;
int g_next = 0;
std::mutex g_mutex;

} // namespace

bool tma_map_for(const double* q, int xc, int yc, int zc, int nvar, int box_x, int box_y, int nv, CUtensorMap* out,
                 int box_z) {
    if ((reinterpret_cast<uintptr_t>(q) & 15) != 0 || (size_t(xc) * 8) % 16 != 0 || box_x > 256 || box_y > 256 ||
        box_z > 256 || nv > 256 || box_x > xc || box_y > yc || box_z > zc || (size_t(box_x) * 8) % 16 != 0 ||
        (zc == 1 && box_z != 1)) {
        return false;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    for (int k = 0; k < g_used; ++k) {
        const Entry& e = g_cache[k];
        if (e.q == q && e.xc == xc && e.yc == yc && e.zc == zc && e.nvar == nvar && e.bx == box_x && e.by == box_y &&
            e.nv == nv && e.bz == box_z) {
            *out = e.map;
            return true;
        }
    }
    PFN_cuTensorMapEncodeTiled fn = encode_fn();
    if (!fn) {
        return false;
    }
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    const cuuint64_t plane = cuuint64_t(xc) * yc * zc;
    CUresult r;
    if (zc == 1) {
        const cuuint64_t dims[3] = {cuuint64_t(xc), cuuint64_t(yc), cuuint64_t(nvar)};
        const cuuint64_t strides[2] = {cuuint64_t(xc) * 8, plane * 8};
        const cuuint32_t box[3] = {cuuint32_t(box_x), cuuint32_t(box_y), cuuint32_t(nv)};
        const cuuint32_t estr[3] = {1, 1, 1};
        r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<double*>(q), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        const cuuint64_t dims[4] = {cuuint64_t(xc), cuuint64_t(yc), cuuint64_t(zc), cuuint64_t(nvar)};
        const cuuint64_t strides[3] = {cuuint64_t(xc) * 8, cuuint64_t(xc) * yc * 8, plane * 8};
        const cuuint32_t box[4] = {cuuint32_t(box_x), cuuint32_t(box_y), cuuint32_t(box_z), cuuint32_t(nv)};
        const cuuint32_t estr[4] = {1, 1, 1, 1};
        r = fn(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double*>(q), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    if (r != CUDA_SUCCESS) {
        return false;
    }
    Entry& e = g_cache[g_next];
    e = Entry{q, xc, yc, zc, nvar, box_x, box_y, nv, box_z, map};
    g_next = (g_next + 1) % kCache;
    if (g_used < kCache) {
        ++g_used;
    }
    *out = map;
    return true;
}

} // namespace mc
