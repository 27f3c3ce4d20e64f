// CSR SpMV, conjugate-gradient solvers and P1 assembly for sm_100a.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "numerics.cuh"

namespace sb {
namespace {

constexpr int kBlock = 256;
constexpr int kGroup = 8;  // lanes per CSR row (~15 nonzeros per row)
constexpr int kRowsPerBlock = kBlock / kGroup;
constexpr int kCgBlocks = kNumSMs * 8;  // 8 resident blocks of 256 threads per SM

template <typename T>
__device__ __forceinline__ double to_d(T v) { return (double)v; }

__device__ __forceinline__ double block_reduce_sum(double v, double* s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < (int)(blockDim.x >> 5) ? s[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    }
    return t;  // thread 0
}

// Row sum of one CSR row by a group of kGroup lanes (result in every lane).
// Every lane of the warp calls it (the shuffles name the full warp); lanes of
// rows past the end (valid false) contribute nothing.
template <typename V, typename X, typename A>
__device__ __forceinline__ A row_dot(uint32_t r, bool valid, const uint32_t* __restrict__ row,
                                     const uint32_t* __restrict__ col, const V* __restrict__ val,
                                     const X* __restrict__ x, int gl) {
    A s = 0;
    if (valid) {
        const uint32_t e = __ldg(&row[r + 1]);
        for (uint32_t j = __ldg(&row[r]) + gl; j < e; j += kGroup) s += (A)__ldg(&val[j]) * (A)__ldg(&x[__ldg(&col[j])]);
    }
#pragma unroll
    for (int o = kGroup / 2; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o, kGroup);
    return s;
}


// L2 eviction policies: the matrix streams through once per product
// (evict_first), the gathered vectors (a few MB) must stay in L2 across the
// whole product (evict_last); without the hints the streamed arrays push the
// vector's sectors out and each is fetched from DRAM several times.
__device__ __forceinline__ uint64_t policy_stream() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_keep() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* a, uint64_t pol) {
    uint32_t v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const float* a, uint64_t pol) {
    float v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_stream(const double* a, uint64_t pol) {
    double v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ float ld_stream(const __half* a, uint64_t pol) {
    unsigned short v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b16 %0, [%1], %2;" : "=h"(v) : "l"(a), "l"(pol));
    return __half2float(__ushort_as_half(v));
}
__device__ __forceinline__ float ld_keep(const float* a, uint64_t pol) {
    float v;
    asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
    return v;
}
__device__ __forceinline__ double ld_keep(const double* a, uint64_t pol) {
    double v;
    asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
    return v;
}

// Dot product of one CSR row (entries b..e) by a group of kLanes lanes, with
// the vector given by gx(column, keep-policy).  Loads go in batches of kBatch
// independent column/value pairs per lane, then their gathers, so that each
// thread keeps several requests in flight.  Every lane of the warp calls it
// (the final shuffles name the whole warp); lanes without a row pass b == e.
template <int kLanes, int kBatch, typename V, typename X, typename Gather>
__device__ __forceinline__ X csr_row(uint32_t b, uint32_t e, int gl, const uint32_t* __restrict__ col,
                                     const V* __restrict__ val, Gather gx) {
    const uint64_t ps = policy_stream(), pk = policy_keep();
    X acc = 0;
    for (uint32_t k0 = b + gl; k0 < e; k0 += kLanes * kBatch) {
        uint32_t c[kBatch];
        X v[kBatch];
#pragma unroll
        for (int u = 0; u < kBatch; ++u) {
            const uint32_t k = k0 + u * kLanes;
            if (k < e) {
                c[u] = ld_stream(&col[k], ps);
                v[u] = (X)ld_stream(&val[k], ps);
            }
        }
#pragma unroll
        for (int u = 0; u < kBatch; ++u)
            if (k0 + u * kLanes < e) acc += v[u] * gx(c[u], pk);
    }
#pragma unroll
    for (int o = kLanes / 2; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o, kLanes);
    return acc;
}

// Lanes per row and batch of the CG products on the 1M-row dam-break matrix
// (A rows hold ~17 entries, the halves of G ~9): A with 4 lanes and batches
// of 5 (FP32, a row in one pass) or 2 (FP64); the halves of G with 2 lanes
// and batches of 4.  Measured against 4 lanes x 4 (FP32) for every product:
// the learned-FSAI solve 30.7 -> 29.5 ms; G with 4 lanes x 3 or 8 x 2 was
// slower (35.2, 38.4 ms).
constexpr int kRowLanes = 4;
constexpr int kGLanes = 2, kGBatch = 4, kGRows = kBlock / kGLanes;
constexpr int kRowsPerBlockCsr = kBlock / kRowLanes;
template <typename X>
constexpr int batch_of() { return sizeof(X) == 8 ? 2 : 5; }

// ---- CG kernels -------------------------------------------------------------
// Mode kRef: the reference's FP32 recurrence (FP32 scalars rounded from
// FP64-accumulated dots, absolute stop sqrt(r.z) <= 1e-6, iteration counter
// of conjugate_gradient.cpp:132).  Otherwise: FP64 scalars, relative stop.
// Iteration k = sc->kbase + kk, kk the position inside a captured batch.

// r = b - A x ; z = M^-1 r ; d = z ; slot0 <- r.z, r.r ; b.b
template <typename V, typename X>
__global__ void __launch_bounds__(kBlock) k_cg_init(uint32_t n, const uint32_t* __restrict__ row,
                                                    const uint32_t* __restrict__ col, const V* __restrict__ val,
                                                    const X* __restrict__ b, const X* __restrict__ x,
                                                    const X* __restrict__ idiag, X* __restrict__ r, X* __restrict__ z,
                                                    X* __restrict__ d, CgScalars* sc, int jacobi) {
    __shared__ double s[32];
    const int gl = threadIdx.x % kGroup;
    double rz = 0.0, rr = 0.0, bb = 0.0;
    for (uint32_t r0 = blockIdx.x * kRowsPerBlock; r0 < n; r0 += gridDim.x * kRowsPerBlock) {
        const uint32_t rid = r0 + threadIdx.x / kGroup;
        const X ax = row_dot<V, X, X>(rid, rid < n, row, col, val, x, gl);
        if (rid < n && gl == 0) {
            const X ri = b[rid] - ax;
            const X zi = jacobi ? ri * idiag[rid] : ri;
            r[rid] = ri;
            z[rid] = zi;
            d[rid] = zi;
            rz += to_d(ri) * to_d(zi);
            rr += to_d(ri) * to_d(ri);
            bb += to_d(b[rid]) * to_d(b[rid]);
        }
    }
    rz = block_reduce_sum(rz, s);
    if (threadIdx.x == 0) atomicAdd(&sc->rz[0], rz);
    rr = block_reduce_sum(rr, s);
    if (threadIdx.x == 0) atomicAdd(&sc->rr[0], rr);
    bb = block_reduce_sum(bb, s);
    if (threadIdx.x == 0) atomicAdd(&sc->bnorm2, bb);
}

// q = A d ; dq += d.q ; zero the accumulators of slot (k+1)&1.
template <typename V, typename X>
__global__ void __launch_bounds__(kBlock) k_cg_spmv(uint32_t n, const uint32_t* __restrict__ row,
                                                    const uint32_t* __restrict__ col, const V* __restrict__ val,
                                                    const X* __restrict__ d, X* __restrict__ q, CgScalars* sc,
                                                    uint32_t kk) {
    if (sc->done) return;
    __shared__ double s[32];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->rz[(kk + 1) & 1] = 0.0;
        sc->rr[(kk + 1) & 1] = 0.0;
    }
    const int gl = threadIdx.x % kGroup;
    double dq = 0.0;
    for (uint32_t r0 = blockIdx.x * kRowsPerBlock; r0 < n; r0 += gridDim.x * kRowsPerBlock) {
        const uint32_t rid = r0 + threadIdx.x / kGroup;
        const X qi = row_dot<V, X, X>(rid, rid < n, row, col, val, d, gl);
        if (rid < n && gl == 0) {
            q[rid] = qi;
            dq += to_d(d[rid]) * to_d(qi);
        }
    }
    dq = block_reduce_sum(dq, s);
    if (threadIdx.x == 0) atomicAdd(&sc->dq[kk & 1], dq);
}


// 16-byte vectors of the CG vector kernels: 4 floats or 2 doubles per load.
template <typename X>
struct Vec16;
template <>
struct Vec16<float> {
    using T = float4;
    static constexpr int N = 4;
};
template <>
struct Vec16<double> {
    using T = double2;
    static constexpr int N = 2;
};
template <typename X>
__device__ __forceinline__ X& lane_of(typename Vec16<X>::T& v, int j) {
    return reinterpret_cast<X*>(&v)[j];
}
template <typename X>
__device__ __forceinline__ X lane_of(const typename Vec16<X>::T& v, int j) {
    return reinterpret_cast<const X*>(&v)[j];
}

// alpha = rz_k / dq ; x += alpha d ; r -= alpha q ; z = M^-1 r ; slot (k+1)&1 <- r.z, r.r
// (16-byte vectors over the first n - n % N entries, the rest one by one)
template <typename X, bool kRef>
__global__ void __launch_bounds__(kBlock) k_cg_update(uint32_t n, X* __restrict__ x, X* __restrict__ r,
                                                      X* __restrict__ z, const X* __restrict__ d,
                                                      const X* __restrict__ q, const X* __restrict__ idiag,
                                                      CgScalars* sc, uint32_t kk, int jacobi) {
    if (sc->done) return;
    __shared__ double s[32];
    X alpha;
    if (kRef) {
        const float sq = (float)sc->rz[kk & 1];
        const float dq = (float)sc->dq[kk & 1];
        alpha = (X)(sq / dq);
    } else {
        alpha = (X)(sc->rz[kk & 1] / sc->dq[kk & 1]);
    }
    using V = typename Vec16<X>::T;
    constexpr int N = Vec16<X>::N;
    double rz = 0.0, rr = 0.0;
    const uint32_t nv = n / N, t0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (uint32_t v = t0; v < nv; v += st) {
        V xv = reinterpret_cast<const V*>(x)[v], rv = reinterpret_cast<const V*>(r)[v];
        const V dv = __ldg(reinterpret_cast<const V*>(d) + v), qv = __ldg(reinterpret_cast<const V*>(q) + v);
        V iv;
        if (jacobi) iv = __ldg(reinterpret_cast<const V*>(idiag) + v);
        V zv;
#pragma unroll
        for (int j = 0; j < N; ++j) {
            lane_of<X>(xv, j) += alpha * lane_of<X>(dv, j);
            const X ri = lane_of<X>(rv, j) - alpha * lane_of<X>(qv, j);
            lane_of<X>(rv, j) = ri;
            const X zi = jacobi ? ri * lane_of<X>(iv, j) : ri;
            lane_of<X>(zv, j) = zi;
            rz += to_d(ri) * to_d(zi);
            rr += to_d(ri) * to_d(ri);
        }
        reinterpret_cast<V*>(x)[v] = xv;
        reinterpret_cast<V*>(r)[v] = rv;
        reinterpret_cast<V*>(z)[v] = zv;
    }
    for (uint32_t i = nv * N + t0; i < n; i += st) {
        const X di = d[i];
        x[i] += alpha * di;
        const X ri = r[i] - alpha * q[i];
        r[i] = ri;
        const X zi = jacobi ? ri * idiag[i] : ri;
        z[i] = zi;
        rz += to_d(ri) * to_d(zi);
        rr += to_d(ri) * to_d(ri);
    }
    rz = block_reduce_sum(rz, s);
    if (threadIdx.x == 0) atomicAdd(&sc->rz[(kk + 1) & 1], rz);
    rr = block_reduce_sum(rr, s);
    if (threadIdx.x == 0) atomicAdd(&sc->rr[(kk + 1) & 1], rr);
}

// beta = rz_{k+1} / rz_k ; d = z + beta d ; convergence test ; zero dq slot k+1.
template <typename X, bool kRef>
__global__ void __launch_bounds__(kBlock) k_cg_dir(uint32_t n, X* __restrict__ d, const X* __restrict__ z,
                                                   CgScalars* sc, uint32_t kk) {
    if (sc->done) return;
    const double rz1 = sc->rz[(kk + 1) & 1], rz0 = sc->rz[kk & 1];
    X beta;
    if (kRef) beta = (X)((float)rz1 / (float)rz0);
    else beta = (X)(rz1 / rz0);
    using V = typename Vec16<X>::T;
    constexpr int N = Vec16<X>::N;
    const uint32_t nv = n / N, t0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (uint32_t v = t0; v < nv; v += st) {
        V dv = reinterpret_cast<const V*>(d)[v];
        const V zv = __ldg(reinterpret_cast<const V*>(z) + v);
#pragma unroll
        for (int j = 0; j < N; ++j) lane_of<X>(dv, j) = lane_of<X>(zv, j) + beta * lane_of<X>(dv, j);
        reinterpret_cast<V*>(d)[v] = dv;
    }
    for (uint32_t j = nv * N + t0; j < n; j += st) d[j] = z[j] + beta * d[j];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        const uint32_t k = sc->kbase + kk;
        sc->dq[(kk + 1) & 1] = 0.0;
        if (kRef) {
            // while (sqrt(sq) > 1e-6f && it++ < 10000): the reference leaves
            // the loop on a NaN r.z too (same counter); here that exit is
            // recorded as a breakdown (3), the counter cap as 2.
            if (!isfinite(rz1)) { sc->it = k; sc->done = 3; }
            else if (!(sqrtf((float)rz1) > 1e-6f)) { sc->it = k; sc->done = 1; }
            else if (!(k < 10000u)) { sc->it = k + 1; sc->done = 2; }
        } else {
            const double rr1 = sc->rr[(kk + 1) & 1];
            if (rr1 <= sc->tol2 * sc->bnorm2) { sc->it = k + 1; sc->done = 1; }
            else if (!isfinite(rr1) || !isfinite(rz1)) { sc->it = k + 1; sc->done = 3; }  // breakdown
            else if (k + 1 >= sc->maxit) { sc->it = k + 1; sc->done = 2; }
        }
    }
}

__global__ void k_cg_batch_end(CgScalars* sc) { sc->kbase += kPollEvery; }

// Fresh scalars for a run: everything zero except the stopping rule.
__global__ void k_cg_reset(CgScalars* sc, double tol2, uint32_t maxit) {
    CgScalars z{};
    z.tol2 = tol2;
    z.maxit = maxit;
    *sc = z;
}

template <typename V, typename X>
__global__ void __launch_bounds__(kBlock) k_jacobi(uint32_t n, const uint32_t* __restrict__ row,
                                                   const uint32_t* __restrict__ col, const V* __restrict__ val,
                                                   X* __restrict__ idiag) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    X v = (X)0;
    for (uint32_t j = row[i]; j < row[i + 1]; ++j)
        if (col[j] == i) { v = (X)1 / (X)val[j]; break; }
    idiag[i] = v;
}

__global__ void k_jacobi_f64_to_f32(uint32_t n, const double* __restrict__ idiag64, float* __restrict__ idiag32) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) idiag32[i] = (float)idiag64[i];
}

// r = b - A x (FP64) ; accumulate r.r and b.b into out[0..1].
__global__ void __launch_bounds__(kBlock) k_residual_f64(uint32_t n, const uint32_t* __restrict__ row,
                                                         const uint32_t* __restrict__ col, const double* __restrict__ val,
                                                         const double* __restrict__ b, const double* __restrict__ x,
                                                         double* __restrict__ r, double* out) {
    __shared__ double s[32];
    const int gl = threadIdx.x % kGroup;
    double rr = 0.0, bb = 0.0;
    for (uint32_t r0 = blockIdx.x * kRowsPerBlock; r0 < n; r0 += gridDim.x * kRowsPerBlock) {
        const uint32_t rid = r0 + threadIdx.x / kGroup;
        const double ax = row_dot<double, double, double>(rid, rid < n, row, col, val, x, gl);
        if (rid < n && gl == 0) {
            const double ri = b[rid] - ax;
            if (r) r[rid] = ri;
            rr += ri * ri;
            bb += b[rid] * b[rid];
        }
    }
    rr = block_reduce_sum(rr, s);
    if (threadIdx.x == 0) atomicAdd(&out[0], rr);
    bb = block_reduce_sum(bb, s);
    if (threadIdx.x == 0) atomicAdd(&out[1], bb);
}

__global__ void k_axpy_f32_into_f64(uint32_t n, double a, const float* __restrict__ e, double* __restrict__ x) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += a * (double)e[i];
}

__global__ void k_scale_f32(uint32_t n, float a, float* __restrict__ v) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] *= a;
}

__global__ void k_f64_to_f32(uint32_t n, const double* __restrict__ a, float* __restrict__ b) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}

// ---- CG products on CSR with a lane group per row -----------------------------------
// q = A d ; dq += d.q ; zero the accumulators of slot (k+1)&1.
template <typename V, typename X>
__global__ void __launch_bounds__(kBlock) k_spmv_csr(uint32_t n, const uint32_t* __restrict__ row,
                                                     const uint32_t* __restrict__ col, const V* __restrict__ val,
                                                     const X* __restrict__ d, X* __restrict__ q, CgScalars* sc,
                                                     uint32_t kk) {
    if (sc->done) return;
    __shared__ double s[32];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        sc->rz[(kk + 1) & 1] = 0.0;
        sc->rr[(kk + 1) & 1] = 0.0;
    }
    const int gl = threadIdx.x % kRowLanes;
    double dq = 0.0;
    for (uint32_t r0 = blockIdx.x * kRowsPerBlockCsr; r0 < n; r0 += gridDim.x * kRowsPerBlockCsr) {
        const uint32_t i = r0 + threadIdx.x / kRowLanes;
        const uint32_t b = i < n ? __ldg(&row[i]) : 0u, e = i < n ? __ldg(&row[i + 1]) : 0u;
        const X qi = csr_row<kRowLanes, batch_of<X>(), V, X>(b, e, gl, col, val,
                                                            [&](uint32_t c, uint64_t pk) { return ld_keep(&d[c], pk); });
        if (i < n && gl == 0) {
            q[i] = qi;
            dq += to_d(d[i]) * to_d(qi);
        }
    }
    dq = block_reduce_sum(dq, s);
    if (threadIdx.x == 0) atomicAdd(&sc->dq[kk & 1], dq);
}

// FSAI: alpha = rz_k / dq_k ; x += alpha d ; r -= alpha q ; slot (k+1)&1 <- r.r
__global__ void __launch_bounds__(kBlock) k_fsai_cg_update(uint32_t n, float* __restrict__ x, float* __restrict__ r,
                                                           const float* __restrict__ d, const float* __restrict__ q,
                                                           CgScalars* sc, uint32_t kk) {
    if (sc->done) return;
    __shared__ double s[32];
    const float alpha = (float)(sc->rz[kk & 1] / sc->dq[kk & 1]);
    double rr = 0.0;
    const uint32_t nv = n / 4, t0 = blockIdx.x * blockDim.x + threadIdx.x, st = gridDim.x * blockDim.x;
    for (uint32_t v = t0; v < nv; v += st) {
        float4 xv = reinterpret_cast<const float4*>(x)[v], rv = reinterpret_cast<const float4*>(r)[v];
        const float4 dv = __ldg(reinterpret_cast<const float4*>(d) + v);
        const float4 qv = __ldg(reinterpret_cast<const float4*>(q) + v);
        xv.x += alpha * dv.x; xv.y += alpha * dv.y; xv.z += alpha * dv.z; xv.w += alpha * dv.w;
        rv.x -= alpha * qv.x; rv.y -= alpha * qv.y; rv.z -= alpha * qv.z; rv.w -= alpha * qv.w;
        reinterpret_cast<float4*>(x)[v] = xv;
        reinterpret_cast<float4*>(r)[v] = rv;
        rr += (double)rv.x * rv.x + (double)rv.y * rv.y + (double)rv.z * rv.z + (double)rv.w * rv.w;
    }
    for (uint32_t i = nv * 4 + t0; i < n; i += st) {
        x[i] += alpha * d[i];
        const float ri = r[i] - alpha * q[i];
        r[i] = ri;
        rr += (double)ri * ri;
    }
    rr = block_reduce_sum(rr, s);
    if (threadIdx.x == 0) atomicAdd(&sc->rr[(kk + 1) & 1], rr);
}

// FSAI: y = G r (compact lower CSR, FP16 values).
__global__ void __launch_bounds__(kBlock) k_fsai_lower(uint32_t n, const uint32_t* __restrict__ lrow,
                                                       const uint32_t* __restrict__ lcol, const __half* __restrict__ lval,
                                                       const float* __restrict__ r, float* __restrict__ y,
                                                       const CgScalars* sc) {
    if (sc->done) return;
    const int gl = threadIdx.x % kGLanes;
    for (uint32_t r0 = blockIdx.x * kGRows; r0 < n; r0 += gridDim.x * kGRows) {
        const uint32_t i = r0 + threadIdx.x / kGLanes;
        const uint32_t b = i < n ? __ldg(&lrow[i]) : 0u, e = i < n ? __ldg(&lrow[i + 1]) : 0u;
        const float yi = csr_row<kGLanes, kGBatch, __half, float>(b, e, gl, lcol, lval,
                                                              [&](uint32_t c, uint64_t pk) { return ld_keep(&r[c], pk); });
        if (i < n && gl == 0) y[i] = yi;
    }
}

// FSAI: z = G^T y (compact upper CSR); slot <- r.z ; d = z when d is non-null.
__global__ void __launch_bounds__(kBlock) k_fsai_upper(uint32_t n, const uint32_t* __restrict__ urow,
                                                       const uint32_t* __restrict__ ucol, const __half* __restrict__ uval,
                                                       const float* __restrict__ y, const float* __restrict__ r,
                                                       float* __restrict__ z, float* __restrict__ d, CgScalars* sc,
                                                       uint32_t slot) {
    if (sc->done) return;
    __shared__ double s[32];
    const int gl = threadIdx.x % kGLanes;
    double rz = 0.0;
    for (uint32_t r0 = blockIdx.x * kGRows; r0 < n; r0 += gridDim.x * kGRows) {
        const uint32_t i = r0 + threadIdx.x / kGLanes;
        const uint32_t b = i < n ? __ldg(&urow[i]) : 0u, e = i < n ? __ldg(&urow[i + 1]) : 0u;
        const float zi = csr_row<kGLanes, kGBatch, __half, float>(b, e, gl, ucol, uval,
                                                              [&](uint32_t c, uint64_t pk) { return ld_keep(&y[c], pk); });
        if (i < n && gl == 0) {
            z[i] = zi;
            if (d) d[i] = zi;
            rz += (double)r[i] * zi;
        }
    }
    rz = block_reduce_sum(rz, s);
    if (threadIdx.x == 0) atomicAdd(&sc->rz[slot & 1], rz);
}

// Start of an inner FP32 solve of A e = rhs, rhs = r64 * scale: r = rhs,
// x = 0, r.r and b.b into slot 0.
__global__ void __launch_bounds__(kBlock) k_inner_init(uint32_t n, const double* __restrict__ r64, double scale,
                                                       float* __restrict__ r, float* __restrict__ x, CgScalars* sc) {
    __shared__ double s[32];
    double rr = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float ri = (float)(r64[i] * scale);
        r[i] = ri;
        x[i] = 0.f;
        rr += (double)ri * ri;
    }
    rr = block_reduce_sum(rr, s);
    if (threadIdx.x == 0) {
        atomicAdd(&sc->rr[0], rr);
        atomicAdd(&sc->bnorm2, rr);
    }
}

// Jacobi start: z = d = idiag r ; rho_0 = r . z.
template <typename X>
__global__ void __launch_bounds__(kBlock) k_jacobi_apply(uint32_t n, const X* __restrict__ r,
                                                         const X* __restrict__ idiag, X* __restrict__ z,
                                                         X* __restrict__ d, CgScalars* sc) {
    __shared__ double s[32];
    double rz = 0.0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const X zi = r[i] * idiag[i];
        z[i] = zi;
        if (d) d[i] = zi;
        rz += to_d(r[i]) * to_d(zi);
    }
    rz = block_reduce_sum(rz, s);
    if (threadIdx.x == 0) atomicAdd(&sc->rz[0], rz);
}

__global__ void k_absmax(uint32_t m, const float* __restrict__ v, float* out) {
    float mx = 0.f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) mx = fmaxf(mx, fabsf(v[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0 && mx > 0.f) atomicMax(reinterpret_cast<unsigned int*>(out), __float_as_uint(mx));
}

// Grids of the grid-stride CG kernels: at most kCgBlocks blocks, so each
// reduction ends in a few hundred atomics instead of one per 32 rows.
int spmv_grid(uint32_t n) { return std::min(kCgBlocks, grid_for(n, kRowsPerBlock)); }
int vec_grid(uint32_t n) { return std::min(kCgBlocks, grid_for(n, kBlock)); }

// One wave of resident blocks of a grid-stride kernel (its occupancy, cached
// per kernel), or fewer when the work is smaller.
template <typename K>
int resident_grid(K kernel, uint32_t work_blocks) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache;
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find((const void*)kernel);
        if (it == cache.end()) {
            SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0));
            cache[(const void*)kernel] = per_sm;
        } else {
            per_sm = it->second;
        }
    }
    return std::max(1, std::min((int)work_blocks, std::max(1, per_sm) * kNumSMs));
}
int row_blocks(uint32_t n) { return grid_for(n, kRowsPerBlockCsr); }

// A batch of kPollEvery CG iterations captured once into a CUDA graph and
// replayed until the device done flag is set (polled after each batch).
class CgBatches {
  public:
    CgBatches() = default;
    CgBatches(const CgBatches&) = delete;
    CgBatches& operator=(const CgBatches&) = delete;
    ~CgBatches() {
        if (exec_) cudaGraphExecDestroy(exec_);
    }
    // enqueue(kk) launches the kernels of iteration kk of the batch.
    template <typename F>
    void capture(F enqueue, uint32_t kernels_per_iter, CgScalars* sc, cudaStream_t s) {
        cudaGraph_t graph = nullptr;
        SB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        cudaError_t err = cudaSuccess;
        for (uint32_t kk = 0; kk < (uint32_t)kPollEvery && err == cudaSuccess; ++kk) {
            enqueue(kk);
            err = cudaGetLastError();
        }
        if (err == cudaSuccess) {
            k_cg_batch_end<<<1, 1, 0, s>>>(sc);
            err = cudaGetLastError();
        }
        const cudaError_t end = cudaStreamEndCapture(s, &graph);
        check(err, "CG batch capture", __FILE__, __LINE__);
        check(end, "cudaStreamEndCapture", __FILE__, __LINE__);
        err = cudaGraphInstantiate(&exec_, graph, 0);
        cudaGraphDestroy(graph);
        check(err, "cudaGraphInstantiate", __FILE__, __LINE__);
        launches_ = kernels_per_iter * kPollEvery + 1;
    }
    bool ready() const { return exec_ != nullptr; }
    // Replays until done or cap bodies; returns the final scalars.
    CgScalars run(CgScalars* sc, uint32_t cap, PinnedWords& pin, cudaStream_t s) {
        CgScalars host{};
        for (uint32_t k = 0;; k += kPollEvery) {
            SB_CUDA(cudaGraphLaunch(exec_, s));
            count_launches(launches_);
            SB_CUDA(cudaMemcpyAsync(pin.h, sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, s));
            SB_CUDA(cudaStreamSynchronize(s));
            std::memcpy(&host, pin.h, sizeof(CgScalars));
            if (host.done || k + kPollEvery >= cap) break;
        }
        return host;
    }

  private:
    cudaGraphExec_t exec_ = nullptr;
    uint32_t launches_ = 0;
};

// Jacobi / plain CG bodies (q = A d ; update ; direction), A in CSR (the
// reference's FP32 solver).
template <typename V, typename X, bool kRef>
void capture_cg(CgBatches& g, uint32_t n, const uint32_t* row, const uint32_t* col, const V* val, X* x, X* r, X* z,
                X* d, X* q, const X* idiag, CgScalars* sc, int jacobi, cudaStream_t s) {
    const int gv = vec_grid(n), gs = spmv_grid(n);
    g.capture([&](uint32_t kk) {
        k_cg_spmv<V, X><<<gs, kBlock, 0, s>>>(n, row, col, val, d, q, sc, kk);
        k_cg_update<X, kRef><<<gv, kBlock, 0, s>>>(n, x, r, z, d, q, idiag, sc, kk, jacobi);
        k_cg_dir<X, kRef><<<gv, kBlock, 0, s>>>(n, d, z, sc, kk);
    }, 3, sc, s);
}

// Jacobi-PCG bodies (q = A d ; update with z = idiag r ; direction), A in CSR.
template <typename V, typename X>
void capture_jacobi(CgBatches& g, const CsrF64& A, const V* val, X* x, X* r, X* z, X* d, X* q, const X* idiag,
                    CgScalars* sc, cudaStream_t s) {
    const uint32_t n = A.n;
    const int gv = vec_grid(n), gs = resident_grid(k_spmv_csr<V, X>, row_blocks(n));
    g.capture([&](uint32_t kk) {
        k_spmv_csr<V, X><<<gs, kBlock, 0, s>>>(n, A.row.ptr, A.col.ptr, val, d, q, sc, kk);
        k_cg_update<X, false><<<gv, kBlock, 0, s>>>(n, x, r, z, d, q, idiag, sc, kk, 1);
        k_cg_dir<X, false><<<gv, kBlock, 0, s>>>(n, d, z, sc, kk);
    }, 3, sc, s);
}

// FSAI-PCG bodies (q = A d ; update ; y = G r ; z = G^T y ; direction), FP32.
void capture_fsai(CgBatches& g, const CsrF64& A, const FsaiOperator& G, float* x, float* r, float* z, float* d,
                  float* q, float* y, CgScalars* sc, cudaStream_t s) {
    const uint32_t n = A.n;
    const int gv = vec_grid(n), gs = resident_grid(k_spmv_csr<float, float>, row_blocks(n));
    const int gl = resident_grid(k_fsai_lower, grid_for(n, kGRows));
    const int gu = resident_grid(k_fsai_upper, grid_for(n, kGRows));
    g.capture([&](uint32_t kk) {
        k_spmv_csr<float, float><<<gs, kBlock, 0, s>>>(n, A.row.ptr, A.col.ptr, A.val32.ptr, d, q, sc, kk);
        k_fsai_cg_update<<<gv, kBlock, 0, s>>>(n, x, r, d, q, sc, kk);
        k_fsai_lower<<<gl, kBlock, 0, s>>>(n, G.lrow, G.lcol, G.lval, r, y, sc);
        k_fsai_upper<<<gu, kBlock, 0, s>>>(n, G.urow, G.ucol, G.uval, y, r, z, nullptr, sc, kk + 1);
        k_cg_dir<float, false><<<gv, kBlock, 0, s>>>(n, d, z, sc, kk);
    }, 5, sc, s);
}

struct EventTimer {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaStream_t s;
    explicit EventTimer(cudaStream_t st) : s(st) {
        SB_CUDA(cudaEventCreate(&e0));
        SB_CUDA(cudaEventCreate(&e1));
        SB_CUDA(cudaEventRecord(e0, s));
    }
    ~EventTimer() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    double stop() {
        SB_CUDA(cudaEventRecord(e1, s));
        SB_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        SB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        return ms;
    }
};


// FP64 residual r = b - A x, returns {||r||, ||b||}.
std::pair<double, double> residual_norms(const CsrF64& A, const double* b, const double* x, double* r,
                                         DeviceBuffer<double>& acc, PinnedWords& pin, cudaStream_t s) {
    SB_CUDA(cudaMemsetAsync(acc.ptr, 0, 2 * sizeof(double), s));
    k_residual_f64<<<spmv_grid(A.n), kBlock, 0, s>>>(A.n, A.row.ptr, A.col.ptr, A.val.ptr, b, x, r, acc.ptr);
    SB_LAUNCH_CHECK();
    double h2[2];
    SB_CUDA(cudaMemcpyAsync(pin.h, acc.ptr, sizeof h2, cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    std::memcpy(h2, pin.h, sizeof h2);
    return {std::sqrt(h2[0]), std::sqrt(h2[1])};
}

}  // namespace

void CsrF64::make_f32(cudaStream_t s) {
    val32.ensure(nnz);
    k_f64_to_f32<<<grid_for(nnz, 256), 256, 0, s>>>(nnz, val.ptr, val32.ptr);
    SB_LAUNCH_CHECK();
    val32_ready = true;
}

void absmax_f32(const float* v, uint32_t m, float* out, cudaStream_t s) {
    SB_CUDA(cudaMemsetAsync(out, 0, sizeof(float), s));
    k_absmax<<<std::min(kCgBlocks, grid_for(m, 256)), 256, 0, s>>>(m, v, out);
    SB_LAUNCH_CHECK();
}

// Rows whose diagonal entry is missing, zero or not finite: the reference's
// Jacobi leaves idiag uninitialised for a row without a diagonal entry
// (preconditioner_jacobi.cpp:43-48) and divides by a zero one.
__global__ void k_bad_diagonal(uint32_t n, const uint32_t* __restrict__ row, const uint32_t* __restrict__ col,
                               const float* __restrict__ val, uint32_t* count) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    bool bad = false;
    if (i < n) {
        bad = true;
        for (uint32_t j = row[i]; j < row[i + 1]; ++j)
            if (col[j] == i) { bad = !(val[j] != 0.0f && isfinite(1.0f / val[j])); break; }
    }
    const uint32_t m = __ballot_sync(0xffffffffu, bad);
    if (m && (threadIdx.x & 31) == 0) atomicAdd(count, (uint32_t)__popc(m));
}

uint32_t count_bad_diagonal(const CsrF32& A, CgWork& w, cudaStream_t s) {
    if (A.n == 0) return 0;
    DeviceBuffer<double>& acc = w.acc;  // one word of scratch, kept in the workspace
    acc.ensure(2);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(acc.ptr);
    SB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t), s));
    k_bad_diagonal<<<grid_for(A.n, 256), 256, 0, s>>>(A.n, A.row.ptr, A.col.ptr, A.val.ptr, cnt);
    SB_LAUNCH_CHECK();
    SB_CUDA(cudaMemcpyAsync(w.pinned.h, cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    return w.pinned.h[0];
}

uint32_t cg_f32_reference(const CsrF32& A, const float* b, float* x, bool jacobi, CgWork& w, cudaStream_t s,
                          uint32_t* done) {
    const uint32_t n = A.n;
    static_assert(sizeof(CgScalars) <= 64 * sizeof(uint32_t), "pinned scratch too small");
    w.sc.ensure(1);
    w.r32.ensure(n); w.z32.ensure(n); w.d32.ensure(n); w.q32.ensure(n); w.idiag32.ensure(n);
    k_cg_reset<<<1, 1, 0, s>>>(w.sc.ptr, 0.0, 10001u);
    SB_LAUNCH_CHECK();
    if (jacobi) {
        k_jacobi<float, float><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A.row.ptr, A.col.ptr, A.val.ptr, w.idiag32.ptr);
        SB_LAUNCH_CHECK();
    }
    k_cg_init<float, float><<<spmv_grid(n), kBlock, 0, s>>>(n, A.row.ptr, A.col.ptr, A.val.ptr, b, x, w.idiag32.ptr,
                                                            w.r32.ptr, w.z32.ptr, w.d32.ptr, w.sc.ptr, jacobi ? 1 : 0);
    SB_LAUNCH_CHECK();
    CgBatches g;
    capture_cg<float, float, true>(g, n, A.row.ptr, A.col.ptr, A.val.ptr, x, w.r32.ptr, w.z32.ptr, w.d32.ptr,
                                   w.q32.ptr, w.idiag32.ptr, w.sc.ptr, jacobi ? 1 : 0, s);
    const CgScalars h = g.run(w.sc.ptr, 10001u, w.pinned, s);
    if (done) *done = h.done;
    return h.it;
}

double relres_f64(const CsrF64& A, const double* b, const double* x, CgWork& w, cudaStream_t s) {
    DeviceBuffer<double>& acc = w.acc;  // kept in the workspace: no allocation per solve
    acc.ensure(2);
    const auto rb = residual_norms(A, b, x, nullptr, acc, w.pinned, s);
    return rb.second > 0 ? rb.first / rb.second : rb.first;
}

SolveReport pcg_f64(const CsrF64& A, const double* b, double* x, double rtol, uint32_t maxit, CgWork& w,
                    cudaStream_t s) {
    const uint32_t n = A.n;
    SolveReport rep;
    EventTimer t(s);
    w.sc.ensure(1);
    w.r.ensure(n); w.z.ensure(n); w.d.ensure(n); w.q.ensure(n); w.idiag.ensure(n);
    k_cg_reset<<<1, 1, 0, s>>>(w.sc.ptr, rtol * rtol, maxit);
    SB_LAUNCH_CHECK();
    k_jacobi<double, double><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A.row.ptr, A.col.ptr, A.val.ptr, w.idiag.ptr);
    SB_LAUNCH_CHECK();
    k_cg_init<double, double><<<spmv_grid(n), kBlock, 0, s>>>(n, A.row.ptr, A.col.ptr, A.val.ptr, b, x, w.idiag.ptr,
                                                              w.r.ptr, w.z.ptr, w.d.ptr, w.sc.ptr, 1);
    SB_LAUNCH_CHECK();
    CgBatches g;
    capture_jacobi<double, double>(g, A, A.val.ptr, x, w.r.ptr, w.z.ptr, w.d.ptr, w.q.ptr, w.idiag.ptr, w.sc.ptr, s);
    const CgScalars h = g.run(w.sc.ptr, maxit, w.pinned, s);
    rep.ms = t.stop();
    rep.iterations = h.it;
    rep.converged = h.done == 1;
    rep.relres = relres_f64(A, b, x, w, s);
    return rep;
}

SolveReport ir_mixed(const CsrF64& A, const double* b, double* x, double rtol, uint32_t maxit, double inner_rtol,
                     CgWork& w, cudaStream_t s) {
    const uint32_t n = A.n;
    SolveReport rep;
    EventTimer t(s);
    if (!A.val32_ready) const_cast<CsrF64&>(A).make_f32(s);
    w.sc.ensure(1);
    w.r.ensure(n); w.idiag.ensure(n);
    w.r32.ensure(n); w.z32.ensure(n); w.d32.ensure(n); w.q32.ensure(n); w.x32.ensure(n); w.idiag32.ensure(n);
    k_jacobi<double, double><<<grid_for(n, kBlock), kBlock, 0, s>>>(n, A.row.ptr, A.col.ptr, A.val.ptr, w.idiag.ptr);
    SB_LAUNCH_CHECK();
    k_jacobi_f64_to_f32<<<grid_for(n, kBlock), kBlock, 0, s>>>(n, w.idiag.ptr, w.idiag32.ptr);
    SB_LAUNCH_CHECK();
    DeviceBuffer<double>& acc = w.acc;  // kept in the workspace: no allocation per solve
    acc.ensure(2);
    CgBatches g;
    uint32_t total = 0;
    double prev = INFINITY;
    for (uint32_t outer = 0;; ++outer) {
        const auto rb = residual_norms(A, b, x, w.r.ptr, acc, w.pinned, s);
        const double rn = rb.first, bn = rb.second;
        rep.outer = outer;
        if (rn <= rtol * bn || total >= maxit || outer >= 50 || !std::isfinite(rn)) {
            rep.converged = rn <= rtol * bn;
            break;
        }
        const double prev_rn = prev;
        prev = rn;
        // FP32 Jacobi-PCG segment on A e = r / ||r|| (r_0 = rhs, z_0 = idiag r_0), reliable updates
        // between segments as in ir_fsai: the first segment starts with d_0 = z_0, later ones keep
        // the search direction (rescaled to the new units).
        const double tol = inner_rtol > 0 ? inner_rtol : std::min(0.5, std::max(kMixedSegment, 0.5 * rtol * bn / rn));
        const bool keep = outer > 0;
        k_cg_reset<<<1, 1, 0, s>>>(w.sc.ptr, tol * tol, maxit - total);
        SB_LAUNCH_CHECK();
        k_inner_init<<<vec_grid(n), kBlock, 0, s>>>(n, w.r.ptr, 1.0 / rn, w.r32.ptr, w.x32.ptr, w.sc.ptr);
        SB_LAUNCH_CHECK();
        k_jacobi_apply<float><<<vec_grid(n), kBlock, 0, s>>>(n, w.r32.ptr, w.idiag32.ptr, w.z32.ptr,
                                                            keep ? nullptr : w.d32.ptr, w.sc.ptr);
        SB_LAUNCH_CHECK();
        if (keep) {
            k_scale_f32<<<grid_for(n, kBlock), kBlock, 0, s>>>(n, (float)(prev_rn / rn), w.d32.ptr);
            SB_LAUNCH_CHECK();
        }
        if (!g.ready())
            capture_jacobi<float, float>(g, A, A.val32.ptr, w.x32.ptr, w.r32.ptr, w.z32.ptr, w.d32.ptr, w.q32.ptr,
                                         w.idiag32.ptr, w.sc.ptr, s);
        const CgScalars hs = g.run(w.sc.ptr, maxit - total, w.pinned, s);
        total += hs.it;
        k_axpy_f32_into_f64<<<grid_for(n, kBlock), kBlock, 0, s>>>(n, rn, w.x32.ptr, x);
        SB_LAUNCH_CHECK();
    }
    rep.ms = t.stop();
    rep.iterations = total;
    rep.relres = relres_f64(A, b, x, w, s);
    return rep;
}

SolveReport ir_fsai(const CsrF64& A, const double* b, double* x, double rtol, uint32_t maxit, double inner_rtol,
                    const FsaiOperator& G, CgWork& w, cudaStream_t s) {
    const uint32_t n = A.n;
    SolveReport rep;
    EventTimer t(s);
    if (!A.val32_ready) const_cast<CsrF64&>(A).make_f32(s);
    w.sc.ensure(1);
    w.r.ensure(n);
    w.r32.ensure(n); w.z32.ensure(n); w.d32.ensure(n); w.q32.ensure(n); w.x32.ensure(n); w.y32.ensure(n);
    DeviceBuffer<double>& acc = w.acc;  // kept in the workspace: no allocation per solve
    acc.ensure(2);
    CgBatches g;
    uint32_t total = 0;
    double prev = INFINITY;
    bool stagnated = false;
    for (uint32_t outer = 0;; ++outer) {
        const auto rb = residual_norms(A, b, x, w.r.ptr, acc, w.pinned, s);
        const double rn = rb.first, bn = rb.second;
        rep.outer = outer;
        if (rn <= rtol * bn) {
            rep.converged = 1;
            break;
        }
        if (!std::isfinite(rn) || !(rn < 0.5 * prev) || total >= maxit || outer >= 50) {
            stagnated = true;
            if (!std::isfinite(rn) || rn > bn) SB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));  // worse than 0
            break;
        }
        const double prev_rn = prev;
        prev = rn;
        // FP32 FSAI-PCG on A e = r / ||r|| (r_0 = rhs, y = G r_0, z_0 = G^T y) until its residual has
        // dropped by the segment target; then x += ||r|| e and the true FP64 residual replaces the
        // recursive one.  The first segment starts with d_0 = z_0; later ones keep the search
        // direction (rescaled to the new units), so the Krylov information is not thrown away at
        // each replacement (reliable updates, Sleijpen and van der Vorst 1996).
        const double tol = inner_rtol > 0 ? inner_rtol : std::min(0.5, std::max(kMixedSegment, 0.5 * rtol * bn / rn));
        const bool keep = outer > 0;
        k_cg_reset<<<1, 1, 0, s>>>(w.sc.ptr, tol * tol, maxit - total);
        SB_LAUNCH_CHECK();
        k_inner_init<<<vec_grid(n), kBlock, 0, s>>>(n, w.r.ptr, 1.0 / rn, w.r32.ptr, w.x32.ptr, w.sc.ptr);
        SB_LAUNCH_CHECK();
        k_fsai_lower<<<resident_grid(k_fsai_lower, grid_for(n, kGRows)), kBlock, 0, s>>>(n, G.lrow, G.lcol, G.lval,
                                                                                   w.r32.ptr, w.y32.ptr, w.sc.ptr);
        SB_LAUNCH_CHECK();
        k_fsai_upper<<<resident_grid(k_fsai_upper, grid_for(n, kGRows)), kBlock, 0, s>>>(
            n, G.urow, G.ucol, G.uval, w.y32.ptr, w.r32.ptr, w.z32.ptr, keep ? nullptr : w.d32.ptr, w.sc.ptr, 0);
        SB_LAUNCH_CHECK();
        if (keep) {  // residual replaced, direction kept (in the new units of r / ||r||)
            k_scale_f32<<<grid_for(n, kBlock), kBlock, 0, s>>>(n, (float)(prev_rn / rn), w.d32.ptr);
            SB_LAUNCH_CHECK();
        }
        if (!g.ready())
            capture_fsai(g, A, G, w.x32.ptr, w.r32.ptr, w.z32.ptr, w.d32.ptr, w.q32.ptr, w.y32.ptr, w.sc.ptr, s);
        const CgScalars hs = g.run(w.sc.ptr, maxit - total, w.pinned, s);
        total += hs.it;
        k_axpy_f32_into_f64<<<grid_for(n, kBlock), kBlock, 0, s>>>(n, rn, w.x32.ptr, x);
        SB_LAUNCH_CHECK();
    }
    if (stagnated) {
        SolveReport fb = pcg_f64(A, b, x, rtol, maxit > total ? maxit - total : 1, w, s);
        total += fb.iterations;
        rep.converged = fb.converged;
        rep.fallback = 1;
    }
    rep.ms = t.stop();
    rep.iterations = total;
    rep.relres = relres_f64(A, b, x, w, s);
    return rep;
}

// ---- P1 assembly -----------------------------------------------------------------
namespace {

constexpr int kMaxRowCols = 128;   // unique columns per row (P1 rows have ~15)
constexpr int kMaxIncident = 256;  // elements per node

__global__ void k_deg(uint32_t ne, const uint4* __restrict__ el, uint32_t* __restrict__ deg) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ne) return;
    const uint4 e = el[t];
    atomicAdd(&deg[e.x], 1u);
    atomicAdd(&deg[e.y], 1u);
    atomicAdd(&deg[e.z], 1u);
    atomicAdd(&deg[e.w], 1u);
}

__global__ void k_fill_inc(uint32_t ne, const uint4* __restrict__ el, const uint32_t* __restrict__ off,
                           uint32_t* __restrict__ cur, uint32_t* __restrict__ inc) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ne) return;
    const uint4 e = el[t];
    inc[off[e.x] + atomicAdd(&cur[e.x], 1u)] = t;
    inc[off[e.y] + atomicAdd(&cur[e.y], 1u)] = t;
    inc[off[e.z] + atomicAdd(&cur[e.z], 1u)] = t;
    inc[off[e.w] + atomicAdd(&cur[e.w], 1u)] = t;
}

// Sort each node's incident-element list (fixes the accumulation order) and
// find its unique columns (node itself + element neighbours), in ascending
// order: their count into cnt[i], the columns into a slot of 1 + 3m entries at
// cols_out + i + 3 off[i], and for each incident element (sorted order) the
// row positions of its four vertices into incpos (bytes; 255: not in the row).
__global__ void __launch_bounds__(128) k_row_pattern(uint32_t n, const uint4* __restrict__ el,
                                                     const uint32_t* __restrict__ off, uint32_t* __restrict__ inc,
                                                     uint32_t* __restrict__ cnt, uint32_t* __restrict__ cols_out,
                                                     uint32_t* __restrict__ incpos, uint32_t* err) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t b = off[i], e = off[i + 1];
    uint32_t* L = inc + b;
    const uint32_t m = e - b;
    if (m > (uint32_t)kMaxIncident) { atomicOr(err, 1u); }
    for (uint32_t a = 1; a < m; ++a) {
        const uint32_t v = L[a];
        uint32_t c = a;
        while (c > 0 && L[c - 1] > v) { L[c] = L[c - 1]; --c; }
        L[c] = v;
    }
    uint32_t cols[kMaxRowCols];
    uint32_t nc = 1;
    cols[0] = i;
    for (uint32_t a = 0; a < m; ++a) {
        const uint4 t = el[L[a]];
        const uint32_t vs[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t v = vs[k];
            uint32_t c = 0;
            while (c < nc && cols[c] < v) ++c;
            if (c < nc && cols[c] == v) continue;
            if (nc >= (uint32_t)kMaxRowCols) { atomicOr(err, 2u); continue; }
            for (uint32_t s2 = nc; s2 > c; --s2) cols[s2] = cols[s2 - 1];
            cols[c] = v;
            ++nc;
        }
    }
    cnt[i] = nc;
    uint32_t* o = cols_out + i + 3 * (size_t)b;  // room for 1 + 3m columns (each element adds at most 3)
    for (uint32_t c = 0; c < nc; ++c) o[c] = cols[c];
    // positions of each incident element's vertices in the row (one byte each, nc <= kMaxRowCols)
    for (uint32_t a = 0; a < m; ++a) {
        const uint4 t = el[L[a]];
        const uint32_t vs[4] = {t.x, t.y, t.z, t.w};
        uint32_t packed = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t lo = 0, hi = nc;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (cols[mid] < vs[k]) lo = mid + 1; else hi = mid;
            }
            packed |= (lo < nc && cols[lo] == vs[k] ? lo : 255u) << (8 * k);
        }
        incpos[b + a] = packed;
    }
}

// Moves row i's columns from their bounded slot (k_row_pattern) to the CSR.
__global__ void k_row_cols(uint32_t n, const uint32_t* __restrict__ off, const uint32_t* __restrict__ tmp,
                           const uint32_t* __restrict__ rowptr, uint32_t* __restrict__ col) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t* src = tmp + i + 3 * (size_t)off[i];
    const uint32_t r0 = rowptr[i], r1 = rowptr[i + 1];
    for (uint32_t c = r0; c < r1; ++c) col[c] = src[c - r0];
}

__device__ __forceinline__ double3 d3(float4 p) { return make_double3(p.x, p.y, p.z); }
__device__ __forceinline__ double3 sub(double3 a, double3 b) { return make_double3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ double3 cross(double3 a, double3 b) {
    return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double dot(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// Row i of the P1 stiffness and load: sum over the incident elements (in
// sorted order) of vol * grad(phi_i) . grad(phi_j), and vol/4 * f(centroid).
__global__ void __launch_bounds__(128) k_row_values(uint32_t n, const float4* __restrict__ cm,
                                                    const uint4* __restrict__ el, const uint32_t* __restrict__ off,
                                                    const uint32_t* __restrict__ inc, const uint32_t* __restrict__ incpos,
                                                    const uint32_t* __restrict__ rowptr,
                                                    const uint32_t* __restrict__ cols, const uint8_t* __restrict__ is_bnd,
                                                    int rhs_kind, DivModes modes, double* __restrict__ val,
                                                    double* __restrict__ b, uint32_t* isolated) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t r0 = rowptr[i], r1 = rowptr[i + 1];
    for (uint32_t c = r0; c < r1; ++c) val[c] = 0.0;
    const bool dir = is_bnd[i] != 0 || off[i + 1] == off[i];
    if (dir) {
        if (!is_bnd[i]) atomicAdd(isolated, 1u);
        for (uint32_t c = r0; c < r1; ++c)
            if (cols[c] == i) val[c] = 1.0;
        b[i] = 0.0;
        return;
    }
    double bi = 0.0;
    for (uint32_t a = off[i]; a < off[i + 1]; ++a) {
        const uint4 t = el[inc[a]];
        const uint32_t v[4] = {t.x, t.y, t.z, t.w};
        const double3 x0 = d3(cm[v[0]]), x1 = d3(cm[v[1]]), x2 = d3(cm[v[2]]), x3 = d3(cm[v[3]]);
        const double3 e1 = sub(x1, x0), e2 = sub(x2, x0), e3 = sub(x3, x0);
        const double det = dot(e1, cross(e2, e3));
        if (det == 0.0) continue;
        const double inv = 1.0 / det;
        double3 g[4];
        g[1] = cross(e2, e3); g[2] = cross(e3, e1); g[3] = cross(e1, e2);
        for (int k = 1; k < 4; ++k) g[k] = make_double3(g[k].x * inv, g[k].y * inv, g[k].z * inv);
        g[0] = make_double3(-(g[1].x + g[2].x + g[3].x), -(g[1].y + g[2].y + g[3].y), -(g[1].z + g[2].z + g[3].z));
        const double vol = fabs(det) / 6.0;
        int li = 0;
        for (int k = 0; k < 4; ++k) if (v[k] == i) li = k;
        const uint32_t pos = incpos[a];
        for (int k = 0; k < 4; ++k) {
            if (is_bnd[v[k]]) continue;  // column elimination (u = 0 there)
            const double kv = vol * dot(g[li], g[k]);
            const uint32_t p = (pos >> (8 * k)) & 0xffu;  // row position of column v[k]
            if (p < r1 - r0) val[r0 + p] += kv;
        }
        double f = 1.0;
        if (rhs_kind == 1) {
            const double cx = 0.25 * (x0.x + x1.x + x2.x + x3.x), cy = 0.25 * (x0.y + x1.y + x2.y + x3.y),
                         cz = 0.25 * (x0.z + x1.z + x2.z + x3.z);
            f = 0.0;
            for (int m = 0; m < modes.count; ++m)
                f += (double)modes.adotk[m] * cos((double)modes.k[m][0] * cx + (double)modes.k[m][1] * cy +
                                                  (double)modes.k[m][2] * cz + (double)modes.phi[m]);
        }
        bi += 0.25 * vol * f;
    }
    b[i] = bi;
}

}  // namespace

void assemble_p1_laplacian(uint32_t n, const float4* cm, const uint4* elems, uint32_t n_elems, const uint8_t* is_bnd,
                           int rhs_kind, const DivModes& modes, CsrF64& A, DeviceBuffer<double>& b, Assembly& asmb,
                           cudaStream_t s) {
    asmb.deg.ensure(n); asmb.off.ensure((size_t)n + 1); asmb.cur.ensure(n); asmb.cnt.ensure(n);
    asmb.inc.ensure((size_t)n_elems * 4);
    DeviceBuffer<uint32_t>& words = asmb.words;
    words.ensure(4);
    SB_CUDA(cudaMemsetAsync(words.ptr, 0, 4 * sizeof(uint32_t), s));
    SB_CUDA(cudaMemsetAsync(asmb.deg.ptr, 0, sizeof(uint32_t) * n, s));
    SB_CUDA(cudaMemsetAsync(asmb.cur.ptr, 0, sizeof(uint32_t) * n, s));
    if (n_elems) {
        k_deg<<<grid_for(n_elems, 256), 256, 0, s>>>(n_elems, elems, asmb.deg.ptr);
        SB_LAUNCH_CHECK();
    }
    exclusive_scan_u32(asmb.scan, asmb.deg.ptr, asmb.off.ptr, n, s);
    if (n_elems) {
        k_fill_inc<<<grid_for(n_elems, 256), 256, 0, s>>>(n_elems, elems, asmb.off.ptr, asmb.cur.ptr, asmb.inc.ptr);
        SB_LAUNCH_CHECK();
    }
    asmb.tmp.ensure((size_t)n + 12 * (size_t)n_elems);
    asmb.incpos.ensure((size_t)n_elems * 4);
    k_row_pattern<<<grid_for(n, 128), 128, 0, s>>>(n, elems, asmb.off.ptr, asmb.inc.ptr, asmb.cnt.ptr, asmb.tmp.ptr,
                                                   asmb.incpos.ptr, words.ptr);
    SB_LAUNCH_CHECK();
    A.n = n;
    A.row.ensure((size_t)n + 1);
    exclusive_scan_u32(asmb.scan, asmb.cnt.ptr, A.row.ptr, n, s);
    uint32_t nnz = 0;
    SB_CUDA(cudaMemcpyAsync(&nnz, A.row.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    A.nnz = nnz;
    A.col.ensure(nnz);
    A.val.ensure(nnz);
    b.ensure(n);
    k_row_cols<<<grid_for(n, 256), 256, 0, s>>>(n, asmb.off.ptr, asmb.tmp.ptr, A.row.ptr, A.col.ptr);
    SB_LAUNCH_CHECK();
    k_row_values<<<grid_for(n, 128), 128, 0, s>>>(n, cm, elems, asmb.off.ptr, asmb.inc.ptr, asmb.incpos.ptr, A.row.ptr,
                                                  A.col.ptr, is_bnd,
                                                  rhs_kind, modes, A.val.ptr, b.ptr, words.ptr + 1);
    SB_LAUNCH_CHECK();
    uint32_t w[2];
    SB_CUDA(cudaMemcpyAsync(w, words.ptr, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    SB_CUDA(cudaStreamSynchronize(s));
    asmb.overflow = w[0];
    asmb.n_isolated = w[1];
    A.invalidate_derived();
}

}  // namespace sb
