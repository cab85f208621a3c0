// Slab decomposition data plane (slab.h): ghost-layer exchange and the
// domain-wide CFL minimum with NCCL, issued from the library in the
// caller's stream. The reference runs one domain (its halo would ride the
// boundary hook it calls after every fill, source/Boundaries.hpp:146-148);
// the exchange here takes that place.
//
// NCCL is loaded at run time (the process's libnccl.so.2 when one is
// already loaded, e.g. by torch, otherwise the first on the library path),
// so the library has no link-time dependency on it.
#include <dlfcn.h>
#include <nccl.h>

#include <cstring>
#include <mutex>
#include <new>

#include "slab.h"

namespace mc {

namespace {

struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId*);
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int);
    ncclResult_t (*comm_destroy)(ncclComm_t);
    ncclResult_t (*group_start)();
    ncclResult_t (*group_end)();
    ncclResult_t (*send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t);
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t, cudaStream_t);
    const char* (*error_string)(ncclResult_t);
};

const NcclApi* nccl_api(const char** err) {
    static NcclApi api;
    static bool ok = false;
    static const char* why = "NCCL not loaded";
    static std::once_flag once;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
        if (!h) {
            h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
        }
        if (!h) {
            why = "cannot load libnccl.so.2";
            return;
        }
        bool all = true;
        auto sym = [&](const char* name) {
            void* p = dlsym(h, name);
            all = all && p != nullptr;
            return p;
        };
        api.get_unique_id = reinterpret_cast<decltype(api.get_unique_id)>(sym("ncclGetUniqueId"));
        api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(sym("ncclCommInitRank"));
        api.comm_destroy = reinterpret_cast<decltype(api.comm_destroy)>(sym("ncclCommDestroy"));
        api.group_start = reinterpret_cast<decltype(api.group_start)>(sym("ncclGroupStart"));
        api.group_end = reinterpret_cast<decltype(api.group_end)>(sym("ncclGroupEnd"));
        api.send = reinterpret_cast<decltype(api.send)>(sym("ncclSend"));
        api.recv = reinterpret_cast<decltype(api.recv)>(sym("ncclRecv"));
        api.all_reduce = reinterpret_cast<decltype(api.all_reduce)>(sym("ncclAllReduce"));
        api.error_string = reinterpret_cast<decltype(api.error_string)>(sym("ncclGetErrorString"));
        if (!all) {
            why = "libnccl.so.2 lacks a symbol the exchange needs";
            return;
        }
        ok = true;
    });
    if (!ok) {
        *err = why;
        return nullptr;
    }
    return &api;
}

} // namespace

struct SlabExchange {
    const NcclApi* api;
    ncclComm_t comm;
    int rank, world;
    int axis;             // 1 (y) or 2 (z)
    int n, ng;            // interior cells along the axis on this rank, ghost layers
    long long plane;      // doubles per variable
    long long layer;      // doubles per layer of the axis (xc, or xc * yc)
    int nvar;
    int below, above;     // neighbour ranks, -1 for none
};

bool slab_unique_id(unsigned char* id, const char** err) {
    const NcclApi* api = nccl_api(err);
    if (!api) {
        return false;
    }
    ncclUniqueId u;
    const ncclResult_t r = api->get_unique_id(&u);
    if (r != ncclSuccess) {
        *err = api->error_string(r);
        return false;
    }
    std::memcpy(id, u.internal, kSlabIdBytes);
    return true;
}

SlabExchange* slab_create(const unsigned char* id, int rank, int world, int axis, int n, int ng, int xc, int yc,
                          int zc, int nvar, bool periodic, const char** err) {
    const NcclApi* api = nccl_api(err);
    if (!api) {
        return nullptr;
    }
    ncclUniqueId u;
    std::memcpy(u.internal, id, kSlabIdBytes);
    SlabExchange* s = new (std::nothrow) SlabExchange();
    if (!s) {
        *err = "host allocation";
        return nullptr;
    }
    s->api = api;
    const ncclResult_t r = api->comm_init_rank(&s->comm, world, u, rank);
    if (r != ncclSuccess) {
        *err = api->error_string(r);
        delete s;
        return nullptr;
    }
    s->rank = rank;
    s->world = world;
    s->axis = axis;
    s->n = n;
    s->ng = ng;
    s->plane = (long long)xc * yc * zc;
    s->layer = axis == 1 ? (long long)xc : (long long)xc * yc;
    s->nvar = nvar;
    s->below = rank > 0 ? rank - 1 : (periodic ? world - 1 : -1);
    s->above = rank < world - 1 ? rank + 1 : (periodic ? 0 : -1);
    return s;
}

void slab_destroy(SlabExchange* s) {
    if (s) {
        s->api->comm_destroy(s->comm);
        delete s;
    }
}

int slab_face_mask(const SlabExchange* s) {
    int m = 0;
    if (s->below >= 0) {
        m |= 1 << (2 * s->axis);
    }
    if (s->above >= 0) {
        m |= 1 << (2 * s->axis + 1);
    }
    return m;
}

// The first ng interior layers [ng, 2 ng) go to the rank below, which puts
// them in its end ghosts [n + ng, n + 2 ng); the last ng interior layers
// [n, n + ng) go to the rank above, into its start ghosts [0, ng). Every
// variable's layers are one contiguous block. Messages travelling down are
// posted before messages travelling up on every rank, so that with two ranks
// (the same peer below and above) or one periodic rank (itself) the sends
// and receives between a pair match in order.
cudaError_t slab_exchange(SlabExchange* s, double* q, cudaStream_t stream, const char** err) {
    const NcclApi& a = *s->api;
    const size_t count = size_t(s->ng) * size_t(s->layer);
    ncclResult_t r = a.group_start();
    for (int v = 0; v < s->nvar && r == ncclSuccess; ++v) {
        double* base = q + (long long)v * s->plane;
        if (s->below >= 0) {
            r = a.send(base + (long long)s->ng * s->layer, count, ncclFloat64, s->below, s->comm, stream);
        }
        if (r == ncclSuccess && s->above >= 0) {
            r = a.recv(base + (long long)(s->n + s->ng) * s->layer, count, ncclFloat64, s->above, s->comm, stream);
        }
    }
    for (int v = 0; v < s->nvar && r == ncclSuccess; ++v) {
        double* base = q + (long long)v * s->plane;
        if (s->above >= 0) {
            r = a.send(base + (long long)s->n * s->layer, count, ncclFloat64, s->above, s->comm, stream);
        }
        if (r == ncclSuccess && s->below >= 0) {
            r = a.recv(base, count, ncclFloat64, s->below, s->comm, stream);
        }
    }
    const ncclResult_t r2 = a.group_end();
    if (r == ncclSuccess) {
        r = r2;
    }
    if (r != ncclSuccess) {
        *err = a.error_string(r);
        return cudaErrorUnknown;
    }
    return cudaSuccess;
}

cudaError_t slab_reduce_min(SlabExchange* s, uint64_t* word, cudaStream_t stream, const char** err) {
    const ncclResult_t r = s->api->all_reduce(word, word, 1, ncclUint64, ncclMin, s->comm, stream);
    if (r != ncclSuccess) {
        *err = s->api->error_string(r);
        return cudaErrorUnknown;
    }
    return cudaSuccess;
}

cudaError_t slab_halo(SlabExchange* s, const double* send_lo, const double* send_hi, double* recv_lo,
                      double* recv_hi, size_t count, cudaStream_t stream, const char** err) {
    const NcclApi& a = *s->api;
    // down first, then up, as in slab_exchange
    ncclResult_t r = a.group_start();
    if (r == ncclSuccess && s->below >= 0) {
        r = a.send(send_lo, count, ncclFloat64, s->below, s->comm, stream);
    }
    if (r == ncclSuccess && s->above >= 0) {
        r = a.recv(recv_hi, count, ncclFloat64, s->above, s->comm, stream);
    }
    if (r == ncclSuccess && s->above >= 0) {
        r = a.send(send_hi, count, ncclFloat64, s->above, s->comm, stream);
    }
    if (r == ncclSuccess && s->below >= 0) {
        r = a.recv(recv_lo, count, ncclFloat64, s->below, s->comm, stream);
    }
    const ncclResult_t r2 = a.group_end();
    if (r == ncclSuccess) {
        r = r2;
    }
    if (r != ncclSuccess) {
        *err = a.error_string(r);
        return cudaErrorUnknown;
    }
    return cudaSuccess;
}

cudaError_t slab_all_reduce(SlabExchange* s, void* buf, size_t count, SlabReduce op, cudaStream_t stream,
                            const char** err) {
    ncclDataType_t type = ncclUint64;
    ncclRedOp_t red = ncclMin;
    if (op == SlabReduce::kSumF64) {
        type = ncclFloat64;
        red = ncclSum;
    } else if (op == SlabReduce::kMinI64) {
        type = ncclInt64;
    }
    const ncclResult_t r = s->api->all_reduce(buf, buf, count, type, red, s->comm, stream);
    if (r != ncclSuccess) {
        *err = s->api->error_string(r);
        return cudaErrorUnknown;
    }
    return cudaSuccess;
}

} // namespace mc
