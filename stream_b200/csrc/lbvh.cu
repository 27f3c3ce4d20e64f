// Karras LBVH build kernels for sm_100a.  Compiled with -fmad=false: the
// reference's box and Morton arithmetic are separate IEEE operations.
#include <cfloat>

#include "lbvh.cuh"

namespace sb {
namespace {

__device__ __forceinline__ int f2ord(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float ord2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

__global__ void k_bbox_init(int* enc) {
    const int t = threadIdx.x;
    if (t < 3) enc[t] = f2ord(FLT_MAX);
    else if (t < 6) enc[t] = f2ord(-FLT_MAX);
}

// Global box of the spheres, radius included (lbvh.hpp:141-175 uses
// Sphere::get_bbox, primitives.hpp:136-141).  Min/max are exact, so the
// atomic combination order does not matter.  A non-finite coordinate or
// radius sets ST_BAD_INPUT in *status (device inputs are not checked on the
// host).
__global__ void __launch_bounds__(256) k_bbox(const float4* __restrict__ s, uint32_t n, int* enc, uint32_t* status) {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    bool bad = false;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = s[i];
        bad |= !(isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(p.w));
        mn[0] = fminf(mn[0], p.x - p.w); mx[0] = fmaxf(mx[0], p.x + p.w);
        mn[1] = fminf(mn[1], p.y - p.w); mx[1] = fmaxf(mx[1], p.y + p.w);
        mn[2] = fminf(mn[2], p.z - p.w); mx[2] = fmaxf(mx[2], p.z + p.w);
    }
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0 && status) atomicOr(status, (uint32_t)ST_BAD_INPUT);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
            mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
        }
    }
    __shared__ float s_mn[8][3], s_mx[8][3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0)
        for (int k = 0; k < 3; ++k) { s_mn[w][k] = mn[k]; s_mx[w][k] = mx[k]; }
    __syncthreads();
    if (threadIdx.x < 3) {
        float a = FLT_MAX, b = -FLT_MAX;
        for (int ww = 0; ww < (int)(blockDim.x >> 5); ++ww) {
            a = fminf(a, s_mn[ww][threadIdx.x]);
            b = fmaxf(b, s_mx[ww][threadIdx.x]);
        }
        atomicMin(&enc[threadIdx.x], f2ord(a));
        atomicMax(&enc[3 + threadIdx.x], f2ord(b));
    }
}

__device__ __forceinline__ uint64_t spread21(uint32_t a) {
    uint64_t x = a & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}
__device__ __forceinline__ uint32_t spread10(uint32_t a) {
    uint32_t x = a & 0x3ffu;
    x = (x | x << 16) & 0x30000ffu;
    x = (x | x << 8) & 0x0300f00fu;
    x = (x | x << 4) & 0x30c30c3u;
    x = (x | x << 2) & 0x9249249u;
    return x;
}

// splitBy2 / encode_magicbits2D (morton.hpp:61-76): 32 bits per axis.
__device__ __forceinline__ uint64_t spread32(uint32_t a) {
    uint64_t x = a;
    x = (x | x << 16) & 0x0000FFFF0000FFFFULL;
    x = (x | x << 8) & 0x00FF00FF00FF00FFULL;
    x = (x | x << 4) & 0x0F0F0F0F0F0F0F0FULL;
    x = (x | x << 2) & 0x3333333333333333ULL;
    x = (x | x << 1) & 0x5555555555555555ULL;
    return x;
}

// Morton codes of the centres (lbvh.hpp:178-213; morton.hpp:27-76) fused with
// the radix sort's digit histograms.  Also decodes the global box.  bits = 64
// is the 2D code (dim = 2: imax = 2^32 per axis, z ignored).
__global__ void __launch_bounds__(256) k_morton_hist(const float4* __restrict__ s, uint32_t n, int bits,
                                                     const int* __restrict__ enc, float* bb_out,
                                                     uint64_t* __restrict__ codes, uint32_t* __restrict__ vals,
                                                     int passes, uint32_t* __restrict__ hist) {
    __shared__ uint32_t s_hist[kSortMaxPasses * 256];
    __shared__ float s_pmin[3], s_f[3];
    for (int i = threadIdx.x; i < kSortMaxPasses * 256; i += blockDim.x) s_hist[i] = 0;
    if (threadIdx.x < 3) {
        const int k = threadIdx.x;
        const float pmin = ord2f(enc[k]), pmax = ord2f(enc[3 + k]);
        const float imax = bits == 30 ? 1024.0f : bits == 64 ? 4294967296.0f : 2097152.0f;
        const float range = pmax - pmin;
        float f = __fdiv_rn(imax, range);
        if (range * f >= imax) f = nextafterf(f, 0.0f);
        s_pmin[k] = pmin;
        s_f[k] = f;
        if (blockIdx.x == 0) { bb_out[k] = pmin; bb_out[3 + k] = pmax; }
    }
    __syncthreads();
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = s[i];
        const uint32_t qx = __float2uint_rz((p.x - s_pmin[0]) * s_f[0]);
        const uint32_t qy = __float2uint_rz((p.y - s_pmin[1]) * s_f[1]);
        uint64_t c;
        if (bits == 64) {
            c = spread32(qx) | (spread32(qy) << 1);
            codes[i] = c;
            vals[i] = i;
            radix_hist_add(s_hist, c, passes);
            continue;
        }
        const uint32_t qz = __float2uint_rz((p.z - s_pmin[2]) * s_f[2]);
        if (bits == 30) c = (uint64_t)(spread10(qx) | (spread10(qy) << 1) | (spread10(qz) << 2));
        else c = spread21(qx) | (spread21(qy) << 1) | (spread21(qz) << 2);
        codes[i] = c;
        vals[i] = i;
        radix_hist_add(s_hist, c, passes);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += blockDim.x)
        if (s_hist[i]) atomicAdd(&hist[i], s_hist[i]);
}

__global__ void __launch_bounds__(256) k_gather(const float4* __restrict__ s, const uint32_t* __restrict__ perm,
                                                uint32_t n, float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __ldg(&s[perm[i]]);
}

// Karras 2012 hierarchy over sorted codes (lbvh.hpp:246-308), including the
// reference's handling of equal codes (clz of zero is 64; no index tie-break).
__global__ void __launch_bounds__(256) k_karras(const uint64_t* __restrict__ m, int n, int32_t* __restrict__ sep,
                                                uint8_t* __restrict__ cil, uint32_t* __restrict__ leaf_parent,
                                                uint32_t* __restrict__ internal_parent, uint32_t* __restrict__ touched) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    touched[i] = 0u;
    const uint64_t mi = m[i];
    const int dp1 = (i + 1 >= n) ? -1 : __clzll(mi ^ m[i + 1]);
    const int dm1 = (i - 1 < 0) ? -1 : __clzll(mi ^ m[i - 1]);
    const int d = (dp1 - dm1 > 0) ? 1 : -1;
    const int dmin = (i - d < n && i - d >= 0) ? __clzll(mi ^ m[i - d]) : -1;
    int lmax = 2;
    while (i + lmax * d >= 0 && i + lmax * d < n && __clzll(mi ^ m[i + lmax * d]) > dmin) lmax *= 2;
    int l = 0;
    for (int t = lmax / 2; t >= 1; t /= 2) {
        const int k = i + (l + t) * d;
        if (k >= 0 && k < n && __clzll(mi ^ m[k]) > dmin) l += t;
    }
    const int j = i + l * d;
    int gamma = (i + j) >> 1;
    const uint64_t mj = m[j];
    if (mi != mj) {
        const int dnode = __clzll(mi ^ mj);
        int s = 0;
        for (int t = (l + 1) / 2; t >= 1; t = (t + 1) / 2) {
            const int k = i + (s + t) * d;
            if (k >= 0 && k < n && __clzll(mi ^ m[k]) > dnode) s += t;
            if (t == 1) break;
        }
        gamma = i + s * d + (d < 0 ? d : 0);
    }
    sep[i] = gamma;
    uint8_t c = 0;
    if (gamma == (i < j ? i : j)) { c |= 1; leaf_parent[gamma] = (uint32_t)i; }
    else internal_parent[gamma] = (uint32_t)i;
    if (gamma + 1 == (i > j ? i : j)) { c |= 2; leaf_parent[gamma + 1] = (uint32_t)i | 0x80000000u; }
    else internal_parent[gamma + 1] = (uint32_t)i | 0x80000000u;
    if (i == 0) internal_parent[0] = (uint32_t)n;
    cil[i] = c;
}

__device__ __forceinline__ NodeBox leaf_box(float4 p, bool fit_point) {
    NodeBox b;
    if (fit_point) {
        b.lo = make_float4(p.x, p.y, p.z, 0.f);
        b.hi = b.lo;
    } else {
        b.lo = make_float4(p.x - p.w, p.y - p.w, p.z - p.w, 0.f);
        b.hi = make_float4(p.x + p.w, p.y + p.w, p.z + p.w, 0.f);
    }
    return b;
}
__device__ __forceinline__ void combine(NodeBox& a, const NodeBox& b) {
    a.lo.x = fminf(a.lo.x, b.lo.x); a.lo.y = fminf(a.lo.y, b.lo.y); a.lo.z = fminf(a.lo.z, b.lo.z);
    a.hi.x = fmaxf(a.hi.x, b.hi.x); a.hi.y = fmaxf(a.hi.y, b.hi.y); a.hi.z = fmaxf(a.hi.z, b.hi.z);
}

// Bottom-up boxes (lbvh.hpp:311-351): the second thread to reach a node
// combines both children and continues upward.  The sibling box written by the
// first thread is read through L2 after the fence/atomic handshake.
__global__ void __launch_bounds__(256) k_fit(const float4* __restrict__ obj_m, uint32_t n, bool fit_point,
                                             const int32_t* __restrict__ sep, const uint8_t* __restrict__ cil,
                                             const uint32_t* __restrict__ leaf_parent,
                                             const uint32_t* __restrict__ internal_parent, uint32_t* touched,
                                             NodeBox* boxes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    NodeBox data = leaf_box(obj_m[i], fit_point);
    uint32_t parent = leaf_parent[i];
    bool right = (parent & 0x80000000u) != 0;
    parent &= 0x7fffffffu;
    uint32_t guard = 0;
    while (parent < n && atom_or_acq_rel(&touched[parent], 1u) != 0u) {
        const uint32_t other = (uint32_t)sep[parent] + (right ? 0u : 1u);
        NodeBox ob;
        if (cil[parent] & (right ? 1 : 2)) {
            ob = leaf_box(obj_m[other], fit_point);
        } else {
            ob.lo = __ldcg(&boxes[other].lo);
            ob.hi = __ldcg(&boxes[other].hi);
        }
        combine(data, ob);
        __stcg(&boxes[parent].lo, data.lo);
        __stcg(&boxes[parent].hi, data.hi);
        const uint32_t pp = internal_parent[parent];
        right = (pp & 0x80000000u) != 0;
        parent = pp & 0x7fffffffu;
        if (++guard > n) break;
    }
}

}  // namespace

void LBVH3D::sort_stage(const float4* d_obj, uint32_t n_, cudaStream_t stream, uint32_t* d_status,
                        StageMarks* prof) {
    if (n_ < 2) throw std::invalid_argument("LBVH3D: needs at least 2 objects");
    n = n_;
    obj_m.ensure((size_t)n + tail);
    codes.ensure(n);
    perm.ensure(n);
    bb_glob.ensure(6);
    bb_enc.ensure(6);
    sort.prepare(n, bits);
    k_bbox_init<<<1, 32, 0, stream>>>(bb_enc.ptr);
    SB_LAUNCH_CHECK();
    int grid = grid_for(n, 256 * 8);
    if (grid > 8 * kNumSMs) grid = 8 * kNumSMs;
    k_bbox<<<grid, 256, 0, stream>>>(d_obj, n, bb_enc.ptr, d_status);
    SB_LAUNCH_CHECK();
    SB_CUDA(cudaMemsetAsync(sort.hist.ptr, 0, sizeof(uint32_t) * sort.passes * 256, stream));
    k_morton_hist<<<grid, 256, 0, stream>>>(d_obj, n, bits, bb_enc.ptr, bb_glob.ptr, codes.ptr, perm.ptr,
                                            sort.passes, sort.hist.ptr);
    SB_LAUNCH_CHECK();
    if (prof) prof->mark_sort();
    radix_sort_pairs(sort, codes.ptr, perm.ptr, n, bits, /*hist_ready=*/true, d_status, stream);
    if (prof) prof->mark_gather();
    k_gather<<<grid_for(n, 256), 256, 0, stream>>>(d_obj, perm.ptr, n, obj_m.ptr);
    SB_LAUNCH_CHECK();
}

void LBVH3D::build(const float4* d_obj, uint32_t n_, cudaStream_t stream, uint32_t* d_status, StageMarks* prof) {
    sort_stage(d_obj, n_, stream, d_status, prof);
    if (prof) prof->mark_hierarchy();
    sep.ensure(n - 1);
    cil.ensure(n - 1);
    leaf_parent.ensure(n);
    internal_parent.ensure(n - 1);
    touched.ensure(n - 1);
    boxes.ensure(n - 1);
    k_karras<<<grid_for(n - 1, 256), 256, 0, stream>>>(codes.ptr, (int)n, sep.ptr, cil.ptr, leaf_parent.ptr,
                                                        internal_parent.ptr, touched.ptr);
    SB_LAUNCH_CHECK();
    k_fit<<<grid_for(n, 256), 256, 0, stream>>>(obj_m.ptr, n, fit_point, sep.ptr, cil.ptr, leaf_parent.ptr,
                                                internal_parent.ptr, touched.ptr, boxes.ptr);
    SB_LAUNCH_CHECK();
}

}  // namespace sb
