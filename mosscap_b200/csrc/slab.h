// Domain decomposition of one problem into slabs along its slowest active
// axis (y in 2D, z in 3D), one slab per rank (one GPU per rank): after
// every stage the ghost layers between slabs are exchanged with NCCL
// point-to-point in the stream, and dt is the all-reduce MIN of the ranks'
// CFL minima in the stream (slab.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace mc {

struct SlabExchange;

// Bytes of the opaque id rank 0 creates and every rank passes to
// slab_create (NCCL's unique id).
constexpr int kSlabIdBytes = 128;

// Fills id with a new communicator id; false (and a message in *err) when
// NCCL cannot be loaded.
bool slab_unique_id(unsigned char* id, const char** err);

// Joins the communicator of `world` ranks (collective: every rank calls
// it). axis: 1 (y) or 2 (z); n: interior cells along it on this rank; the
// state is nvar x zc x yc x xc doubles. periodic: the outer faces of the
// global problem are periodic, so rank 0 and rank world-1 are neighbours.
SlabExchange* slab_create(const unsigned char* id, int rank, int world, int axis, int n, int ng, int xc, int yc,
                          int zc, int nvar, bool periodic, const char** err);
void slab_destroy(SlabExchange* s);

// Faces (bit f = face f of mc_grid.bc) whose ghost layers the exchange
// fills: the slab axis's start face when the rank has a neighbour below,
// its end face when it has one above.
int slab_face_mask(const SlabExchange* s);

// Enqueue on `stream` the exchange of q's ghost layers along the slab axis.
cudaError_t slab_exchange(SlabExchange* s, double* q, cudaStream_t stream, const char** err);

// Enqueue on `stream` the all-reduce MIN of the 64-bit word holding the bits
// of this rank's non-negative CFL minimum (integer order = value order).
cudaError_t slab_reduce_min(SlabExchange* s, uint64_t* word, cudaStream_t stream, const char** err);

// Enqueue on `stream` one exchange of contiguous blocks of `count` doubles
// with the neighbours along the slab axis: send_lo goes to the rank below
// (into its recv_hi), send_hi to the rank above (into its recv_lo). A side
// with no neighbour sends and receives nothing.
cudaError_t slab_halo(SlabExchange* s, const double* send_lo, const double* send_hi, double* recv_lo,
                      double* recv_hi, size_t count, cudaStream_t stream, const char** err);

// In-place all-reduce of `count` elements over the ranks, in `stream`.
enum class SlabReduce { kMinU64, kSumF64, kMinI64 };
cudaError_t slab_all_reduce(SlabExchange* s, void* buf, size_t count, SlabReduce op, cudaStream_t stream,
                            const char** err);

} // namespace mc
