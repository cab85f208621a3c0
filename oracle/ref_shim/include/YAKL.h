// Oracle test infrastructure, not product code.
//
// Host-only stand-in for the small part of the Kokkos and YAKL APIs that
// Mosscap's hydro hot path uses (source/Types.hpp, source/LoopUtils.hpp,
// source/State.hpp, source/Eos.hpp, source/Reconstruct.hpp,
// source/Riemann.hpp, source/Hydro.cpp, source/TimeStepping.cpp,
// source/Boundaries.hpp, source/SourceTerms.hpp). It lets those files compile
// unmodified with g++ -fopenmp so that the reference's own arithmetic can be
// run on the CPU as the correctness oracle and as the CPU baseline.
//
// The shim supplies containers and loops only; it contributes no arithmetic
// to the hydro path. Semantics follow the public Kokkos/YAKL documentation:
//  - yakl::Array: reference-counted, row-major ("C" style), shallow copies,
//    operator() const returns a mutable reference, deep_copy_to copies data,
//    assignment from a scalar fills.
//  - yakl::SArray: fixed-size value array with mutable storage.
//  - Kokkos::parallel_for / parallel_reduce over a flat index range, run with
//    OpenMP; Kokkos::Min joins with `src < dest ? src : dest` starting from the
//    reduction identity (the largest finite value).
//  - yakl::Array(label, pointer, dims...) wraps memory it does not own.
//
// With MOSSCAP_SHIM_MANAGED defined, memDevice arrays are allocated as CUDA
// managed memory, which a GPU kernel and the host loops can both address:
// the arrays of a Simulation are then device memory, as in Mosscap's CUDA
// build, so the C++ hook adapter can be run against the reference's own
// Simulation type (the adapter check in oracle/adapter_check.cpp).
#pragma once

#ifdef MOSSCAP_SHIM_MANAGED
#include <cuda_runtime.h>
#include <cstdio>
#include <cstdlib>
#endif

#include <atomic>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>

#define KOKKOS_INLINE_FUNCTION inline
#define KOKKOS_FORCEINLINE_FUNCTION inline
#define KOKKOS_FUNCTION
#define KOKKOS_LAMBDA [=]
#define KOKKOS_CLASS_LAMBDA [=, *this]
#define KOKKOS_ASSERT(x) ((void)0)
#define YAKL_INLINE inline
#define YAKL_LAMBDA [=]

namespace Kokkos {

template <class T, std::size_t N>
struct Array {
    T m_data[N];
    KOKKOS_INLINE_FUNCTION T& operator[](std::size_t i) { return m_data[i]; }
    KOKKOS_INLINE_FUNCTION const T& operator[](std::size_t i) const { return m_data[i]; }
    static constexpr std::size_t size() { return N; }
};

struct LayoutRight {};
struct HostSpace {};
enum MemoryTraitsFlags : unsigned { Unmanaged = 1 };
template <unsigned Flags>
struct MemoryTraits {};
template <class T, class... Args>
struct View {};

struct HostOpenMPSpace {
    using memory_space = HostSpace;
    using scratch_memory_space = HostSpace;
    using execution_space = HostOpenMPSpace;
};
using DefaultExecutionSpace = HostOpenMPSpace;
using DefaultHostExecutionSpace = HostOpenMPSpace;

template <class Space = DefaultExecutionSpace>
struct TeamPolicy {
    struct member_type {};
};

template <class Space = DefaultExecutionSpace>
struct RangePolicy {
    int64_t begin;
    int64_t end;
    RangePolicy(int64_t b, int64_t e) : begin(b), end(e) {}
};

template <class T1, class T2>
struct pair {
    T1 first;
    T2 second;
};
template <class T1, class T2>
KOKKOS_INLINE_FUNCTION pair<T1, T2> make_pair(T1 a, T2 b) {
    return pair<T1, T2>{a, b};
}

template <class T>
struct reduction_identity;
template <>
struct reduction_identity<double> {
    static double min() { return DBL_MAX; }
};
template <>
struct reduction_identity<float> {
    static float min() { return FLT_MAX; }
};

template <class Scalar, class Space = HostSpace>
struct Min {
    using value_type = Scalar;
    value_type& ref;
    explicit Min(value_type& r) : ref(r) {}
    static value_type init() { return reduction_identity<Scalar>::min(); }
    static void join(value_type& dest, const value_type& src) {
        dest = (src < dest) ? src : dest;
    }
};

inline void fence() {}

template <class ExecSpace = DefaultExecutionSpace, class F>
void parallel_for(const std::string&, int64_t n, const F& f) {
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        f(i);
    }
}

template <class ExecSpace = DefaultExecutionSpace, class Space, class F>
void parallel_for(const std::string& name, const RangePolicy<Space>& p, const F& f) {
#pragma omp parallel for schedule(static)
    for (int64_t i = p.begin; i < p.end; ++i) {
        f(i);
    }
}

template <class Space, class F, class Reducer>
void parallel_reduce(const RangePolicy<Space>& p, const F& f, const Reducer& r) {
    using V = typename Reducer::value_type;
    V result = Reducer::init();
#pragma omp parallel
    {
        V local = Reducer::init();
#pragma omp for schedule(static) nowait
        for (int64_t i = p.begin; i < p.end; ++i) {
            f(i, local);
        }
#pragma omp critical
        Reducer::join(result, local);
    }
    r.ref = result;
}

// Kokkos::abort stand-in: the oracle must not end the test process, so a
// call is counted (moracle_abort_count) and the calling loop body goes on.
inline std::atomic<long long>& abort_count() {
    static std::atomic<long long> n{0};
    return n;
}
inline void abort(const char*) {
    abort_count().fetch_add(1);
}

} // namespace Kokkos

namespace yakl {

constexpr int memDevice = 1;
constexpr int memHost = 2;
constexpr int styleC = 1;

template <class T>
struct DimsT {
    template <class X>
    explicit DimsT(const X&) {}
};

// NetCDF reader stand-in: the oracle never reads files (its EOS tables are
// set in code), so every call is a no-op.
constexpr int NETCDF_MODE_READ = 0;
constexpr int NETCDF_MODE_WRITE = 1;
struct SimpleNetCDF {
    void open(const std::string&, int) {}
    void close() {}
    template <class T>
    void read(T&, const std::string&) {}
};

inline void timer_start(const std::string&) {}
inline void timer_stop(const std::string&) {}

template <class T, int rank, int myMem, int myStyle = styleC>
class Array {
    using NC = std::remove_const_t<T>;
    std::shared_ptr<NC[]> owner_;
    T* ptr_ = nullptr;
    int64_t dims_[rank] = {};
    std::string label_;

public:
    Array() = default;

    template <class... Ints, std::enable_if_t<sizeof...(Ints) == rank, int> = 0>
    Array(const char* label, Ints... n) : label_(label) {
        const int64_t d[rank] = {int64_t(n)...};
        int64_t total = 1;
        for (int i = 0; i < rank; ++i) {
            dims_[i] = d[i];
            total *= d[i];
        }
#ifdef MOSSCAP_SHIM_MANAGED
        if (myMem == memDevice) {
            NC* p = nullptr;
            if (cudaMallocManaged(reinterpret_cast<void**>(&p), sizeof(NC) * (total > 0 ? total : 1)) !=
                cudaSuccess) {
                std::fprintf(stderr, "yakl shim: cudaMallocManaged failed for %s\n", label);
                std::abort();
            }
            std::memset(static_cast<void*>(p), 0, sizeof(NC) * total);
            owner_ = std::shared_ptr<NC[]>(p, [](NC* x) { cudaFree(x); });
            ptr_ = owner_.get();
            return;
        }
#endif
        owner_ = std::shared_ptr<NC[]>(new NC[total]());
        ptr_ = owner_.get();
    }

    // A view of memory the array does not own (YAKL's unmanaged form).
    template <class... Ints, std::enable_if_t<sizeof...(Ints) == rank, int> = 0>
    Array(const char* label, T* data, Ints... n) : ptr_(data), label_(label) {
        const int64_t d[rank] = {int64_t(n)...};
        for (int i = 0; i < rank; ++i) {
            dims_[i] = d[i];
        }
    }

    template <class... Ints>
    KOKKOS_INLINE_FUNCTION T& operator()(Ints... idx) const {
        static_assert(sizeof...(Ints) == rank, "index rank mismatch");
        const int64_t id[rank] = {int64_t(idx)...};
        int64_t flat = id[0];
        for (int i = 1; i < rank; ++i) {
            flat = flat * dims_[i] + id[i];
        }
        return ptr_[flat];
    }

    int64_t extent(int i) const { return dims_[i]; }
    int64_t size() const {
        int64_t total = 1;
        for (int i = 0; i < rank; ++i) {
            total *= dims_[i];
        }
        return ptr_ ? total : 0;
    }
    T* data() const { return ptr_; }
    bool initialized() const { return ptr_ != nullptr; }
    std::string label() const { return label_; }

    template <class U>
    void deep_copy_to(const Array<U, rank, myMem, myStyle>& other) const {
        std::memcpy((void*)other.data(), (const void*)ptr_, sizeof(T) * size());
    }

    Array& operator=(const Array&) = default;
    Array(const Array&) = default;

    const Array& operator=(NC v) const {
        const int64_t n = size();
        for (int64_t i = 0; i < n; ++i) {
            ptr_[i] = v;
        }
        return *this;
    }
};

template <class T, int rank, unsigned D0, unsigned D1 = 1, unsigned D2 = 1, unsigned D3 = 1>
class SArray {
    mutable T data_[D0 * D1 * D2 * D3];

public:
    SArray() = default;
    explicit SArray(T v) {
        for (unsigned i = 0; i < D0 * D1 * D2 * D3; ++i) {
            data_[i] = v;
        }
    }
    KOKKOS_INLINE_FUNCTION T& operator()(int i) const { return data_[i]; }
    KOKKOS_INLINE_FUNCTION T& operator()(int i, int j) const { return data_[i * D1 + j]; }
    KOKKOS_INLINE_FUNCTION T& operator()(int i, int j, int k) const {
        return data_[(i * D1 + j) * D2 + k];
    }
};

} // namespace yakl
