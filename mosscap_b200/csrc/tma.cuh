// Tensor-memory-accelerator (TMA) tile loads of the conserved state.
//
// The tiled stage kernels stage the haloed tile of Q that a CTA converts to
// primitives with one cp.async.bulk.tensor copy into shared memory (every
// CTA loads its own tile, from this GPU's memory only), completed on an
// mbarrier, instead of one global load per thread, cell and variable.
//
// Device side: mbarrier set-up, the tensor copy and a bounded wait. Host
// side (tma_map_for): the tensor map of a state array, encoded with the
// driver's cuTensorMapEncodeTiled (looked up through the runtime, so the
// library does not link libcuda) and cached per array.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace mc {

// Shared-memory address (32-bit, shared window) of a generic pointer.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
    // make the initialisation visible to the asynchronous (TMA) proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(mbar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_addr(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of the barrier, giving up after `limit` polls
// (each poll may suspend the thread for a short, hardware-chosen time).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* mbar, uint32_t parity, int limit) {
    for (int it = 0; it < limit; ++it) {
        if (mbar_try_wait(mbar, parity)) {
            return true;
        }
    }
    return false;
}

// 3D / 4D tiled tensor copy global -> shared, completing on mbar. The
// innermost coordinate x must be a multiple of 16 bytes' worth of elements
// (even for doubles); the host only builds maps whose tiles start there.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(mbar))
        : "memory");
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint64_t* mbar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_addr(mbar))
        : "memory");
}

// Polls of a TMA completion wait before the kernel gives up and raises
// MC_FLAG_TIMEOUT (far beyond any copy's latency).
constexpr int kTmaWaitPolls = 1 << 20;

// Host: the tensor map of state array q ([nvar][zc][yc][xc] doubles) whose
// box is box_x x box_y x box_z cells (x, y, z), nv variables; the tensor is
// 3D (x, y, var) when zc == 1, else 4D (x, y, z, var). Returns false (and
// the caller falls back to per-thread loads) when the array cannot be
// described: base not 16-byte aligned, a row pitch that is not a multiple of
// 16 bytes, a box larger than the array, or the driver refuses the map.
bool tma_map_for(const double* q, int xc, int yc, int zc, int nvar, int box_x, int box_y, int nv, CUtensorMap* out,
                 int box_z = 1);

} // namespace mc
