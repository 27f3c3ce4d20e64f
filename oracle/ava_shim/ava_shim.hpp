// CPU (OpenMP) stand-in for the subset of the AVA portability layer that the
// reference's PFEM remesh-and-solve sources use.  Test infrastructure only:
// it exists so that the reference's own, unmodified sources
// (include/geometry/lbvh.hpp, src/mesh/DirectAlphaShape3D.cpp,
// src/numerics/*.cpp) compile for the host and can be run as the oracle.
//
// The AVA library itself (deps/ava, an empty git submodule in the reference)
// is not available.  Only the semantics the reference relies on are provided:
//   * AvaDeviceArray / AvaHostArray / AvaView containers (host memory here;
//     rank-1 views and row-major views with a fixed inner extent),
//   * ava_for<B>(stream, smem, n, f): f(i) for i in [0, n), OpenMP parallel,
//   * ava::sort::sort_pairs: stable ascending sort of (key, value) pairs,
//   * ava::scan::{inclusive_sum, inplace_inclusive_sum}: exact integer scans,
//   * ava::reduce::{transform_reduce, sum},
//   * ava::atomic::{fetch_add, fetch_or} with sequentially consistent order,
//   * ava::bits::{clz, ctz} (CUDA semantics at 0), ava::select::flagged (in place),
//   * deep_copy / gpu_memset / ava_device_sync / ERRCHK.
// Call sites: include/geometry/lbvh.hpp:141-243,311-351;
// src/mesh/DirectAlphaShape3D.cpp:235-292,367,697-704; src/mesh/mesh.cpp;
// include/geometry/lbvh_agglo.hpp;
// src/numerics/conjugate_gradient.cpp:44-59.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <initializer_list>
#include <memory>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef AVA_BLOCK_SIZE
#define AVA_BLOCK_SIZE 256
#endif

#ifndef ERRCHK
#define ERRCHK(x) (void)(x)
#endif

// CUDA's clz of zero is 64; the host builtin is undefined there.  The reference
// relies on clz(0) == 64 for duplicate Morton codes (lbvh.hpp:257-258).
static inline int ava_shim_clzll(unsigned long long x) {
    return x == 0ULL ? 64 : __builtin_clzll(x);
}

static inline void __threadfence() { __atomic_thread_fence(__ATOMIC_SEQ_CST); }

// ----------------------------------------------------------------- views ---
template <typename T, int Rank, int Inner = 0>
struct AvaView;

template <typename T>
struct AvaView<T, -1, 0> {
    T* data = nullptr;
    int dyn_shape[1] = {0};
    AvaView() = default;
    AvaView(T* p, const int shape[1]) : data(p) { dyn_shape[0] = shape[0]; }
    T& operator()(long long i) const { return data[i]; }
};

// Row-major view with a fixed inner extent (AvaView<T, -1, 2>: rows of 2,
// include/geometry/lbvh_agglo.hpp:276-277).
template <typename T, int Inner>
struct AvaView<T, -1, Inner> {
    T* data = nullptr;
    int dyn_shape[2] = {0, Inner};
    AvaView() = default;
    AvaView(T* p, const int shape[1]) : data(p) { dyn_shape[0] = shape[0] / Inner; }
    T& operator()(long long i, long long j) const { return data[i * Inner + j]; }
};

// ------------------------------------------------------------ host array ---
template <typename T, typename I = int>
struct AvaHostArray {
    std::vector<T> buf;

    struct Ptr {
        std::shared_ptr<AvaHostArray> p;
        AvaHostArray* operator->() const { return p.get(); }
        AvaHostArray& operator*() const { return *p; }
        T& operator()(long long i) const { return p->buf[i]; }
    };

    static Ptr create(std::initializer_list<I> dims) {
        Ptr r{std::make_shared<AvaHostArray>()};
        size_t n = 1;
        for (I d : dims) n *= (size_t)d;
        r.p->buf.resize(n);
        return r;
    }
    void resize(std::initializer_list<I> dims) {
        size_t n = 1;
        for (I d : dims) n *= (size_t)d;
        buf.resize(n);
    }
    I size() const { return (I)buf.size(); }
    T* data() { return buf.data(); }
    const T* data() const { return buf.data(); }
};

// ---------------------------------------------------------- device array ---
template <typename T, typename I = int>
struct AvaDeviceArray {
    T* data = nullptr;
    I size = 0;
    std::vector<T> store;

    struct Ptr {
        std::shared_ptr<AvaDeviceArray> p;
        AvaDeviceArray* operator->() const { return p.get(); }
        AvaDeviceArray& operator*() const { return *p; }
    };

    static Ptr create(std::initializer_list<I> dims) {
        Ptr r{std::make_shared<AvaDeviceArray>()};
        r.p->resize(dims);
        return r;
    }
    void resize(std::initializer_list<I> dims) {
        size_t n = 1;
        for (I d : dims) n *= (size_t)d;
        // Growth keeps existing contents, like a device realloc + copy.  The
        // store is padded by 512 bytes, as cudaMalloc rounds every allocation
        // up: the reference's LBVHa clears d_touched for tid < n although it
        // allocates n - 1 entries (include/geometry/lbvh_agglo.hpp:143, 263),
        // and on a GPU that one-past-the-end write lands in the rounding.
        store.resize(n + (512 + sizeof(T) - 1) / sizeof(T));
        data = store.data();
        size = (I)n;
    }
    template <int R, int Inner = 0>
    AvaView<T, R, Inner> to_view() const {
        int shape[1] = {(int)size};
        return AvaView<T, R, Inner>(const_cast<T*>(data), shape);
    }
    template <typename HostPtr>
    void set(const HostPtr& h) {
        std::memcpy(data, h->data(), sizeof(T) * (size_t)h->size());
    }
    void set_scalar(T v) { std::fill(store.begin(), store.end(), v); }
};

template <typename T>
static inline void deep_copy(T* dst, const T* src, size_t n) {
    std::memcpy((void*)dst, (const void*)src, n * sizeof(T));
}

template <typename T>
static inline void gpu_memset(T* dst, int v, size_t n) {
    std::memset((void*)dst, v, n * sizeof(T));
}

static inline void ava_device_sync() {}

// ------------------------------------------------------------- ava_for ---
template <int B, typename F>
static inline void ava_for(void* /*stream*/, size_t /*smem*/, size_t n, F f) {
    const long long nn = (long long)n;
#pragma omp parallel for schedule(dynamic, 256)
    for (long long i = 0; i < nn; ++i) f(i);
}

namespace ava {
namespace atomic {
template <typename T>
static inline T fetch_add(T* p, T v) { return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST); }
template <typename T>
static inline T fetch_or(T* p, T v) { return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST); }
}  // namespace atomic

namespace sort {
// Stable ascending sort of (key, value) pairs.  A null tmp is a size query.
template <typename K, typename V>
static inline int sort_pairs(void* tmp, size_t& tmp_size, const K* kin, K* kout,
                             const V* vin, V* vout, size_t n) {
    if (tmp == nullptr) { tmp_size = 16; return 0; }
    std::vector<size_t> idx(n);
    std::iota(idx.begin(), idx.end(), (size_t)0);
    std::stable_sort(idx.begin(), idx.end(),
                     [&](size_t a, size_t b) { return kin[a] < kin[b]; });
    std::vector<K> kt(n);
    std::vector<V> vt(n);
    for (size_t i = 0; i < n; ++i) { kt[i] = kin[idx[i]]; vt[i] = vin[idx[i]]; }
    std::copy(kt.begin(), kt.end(), kout);
    std::copy(vt.begin(), vt.end(), vout);
    return 0;
}
}  // namespace sort

namespace scan {
template <typename T, typename U>
static inline int inclusive_sum(void* tmp, size_t& tmp_size, const T* in, U* out, size_t n) {
    if (tmp == nullptr) { tmp_size = 16; return 0; }
    U acc = 0;
    for (size_t i = 0; i < n; ++i) { acc += (U)in[i]; out[i] = acc; }
    return 0;
}
template <typename T>
static inline int inplace_inclusive_sum(void* tmp, size_t& tmp_size, T* data, size_t n) {
    if (tmp == nullptr) { tmp_size = 16; return 0; }
    T acc = 0;
    for (size_t i = 0; i < n; ++i) { acc += data[i]; data[i] = acc; }
    return 0;
}
}  // namespace scan

namespace bits {
// CUDA semantics: __clz / ctz of 0 is the bit width (src/mesh/mesh.cpp:244-245).
static inline uint32_t clz(uint32_t x) { return x ? (uint32_t)__builtin_clz(x) : 32u; }
static inline uint32_t ctz(uint32_t x) { return x ? (uint32_t)__builtin_ctz(x) : 32u; }
static inline uint32_t clz(uint64_t x) { return x ? (uint32_t)__builtin_clzll(x) : 64u; }
static inline uint32_t ctz(uint64_t x) { return x ? (uint32_t)__builtin_ctzll(x) : 64u; }
}  // namespace bits

namespace select {
// In-place stable compaction of data[i] with flags[i] != 0 (CUB
// DeviceSelect::Flagged's in-place form; src/mesh/mesh.cpp:601-627).  data and
// flags may be the same array.
template <typename T, typename F, typename N>
static inline int flagged(void* tmp, size_t& tmp_size, T* data, const F* flags, N* num_selected, size_t n) {
    if (tmp == nullptr) { tmp_size = 16; return 0; }
    size_t k = 0;
    for (size_t i = 0; i < n; ++i) {
        const bool keep = flags[i] != 0;
        if (keep) data[k++] = data[i];
    }
    *num_selected = (N)k;
    return 0;
}
}  // namespace select

namespace reduce {
template <typename In, typename Out, typename R, typename Tr, typename Init>
static inline int transform_reduce(void* tmp, size_t& tmp_size, const In* in, Out* out,
                                   size_t n, R red, Tr tr, Init init) {
    if (tmp == nullptr) { tmp_size = 16; return 0; }
    Out acc = init;
    for (size_t i = 0; i < n; ++i) acc = red(acc, tr(in[i]));
    *out = acc;
    return 0;
}
// Pairwise (tree) summation, the shape of a device-wide reduction.
template <typename T>
static inline T pairwise_sum(const T* in, size_t n) {
    if (n <= 8) { T s = 0; for (size_t i = 0; i < n; ++i) s += in[i]; return s; }
    size_t h = n / 2;
    return pairwise_sum(in, h) + pairwise_sum(in + h, n - h);
}
template <typename T>
static inline int sum(void* /*tmp*/, size_t /*tmp_size*/, const T* in, T* out, size_t n) {
    *out = pairwise_sum(in, n);
    return 0;
}
}  // namespace reduce
}  // namespace ava
