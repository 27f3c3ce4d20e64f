// TRBVH kernels for sm_100a (compiled with -fmad=false: SAH sums and areas are
// separate IEEE operations so results are reproducible operation by operation).
#include <cfloat>

#include "trbvh.cuh"

namespace sb {
namespace {

constexpr float kCi = 1.2f;  // trbvh.hpp:72
constexpr float kCt = 1.0f;  // trbvh.hpp:73

__device__ __forceinline__ float area_of(const NodeBox& b, bool area3d) {
    const float ex = b.hi.x - b.lo.x, ey = b.hi.y - b.lo.y, ez = b.hi.z - b.lo.z;
    return area3d ? (ex * ey + ey * ez) + ez * ex : ex * ey;
}
// Ci * A(node) of the Apetrei build: in the 2D measure the reference forms it
// left to right, (Ci * ext_x) * ext_y (trbvh.hpp:373).
__device__ __forceinline__ float ci_area_of(const NodeBox& b, bool area3d) {
    const float ex = b.hi.x - b.lo.x, ey = b.hi.y - b.lo.y;
    return area3d ? kCi * area_of(b, true) : (kCi * ex) * ey;
}
__device__ __forceinline__ void box_union(NodeBox& a, const NodeBox& b) {
    a.lo.x = fminf(a.lo.x, b.lo.x); a.lo.y = fminf(a.lo.y, b.lo.y); a.lo.z = fminf(a.lo.z, b.lo.z);
    a.hi.x = fmaxf(a.hi.x, b.hi.x); a.hi.y = fmaxf(a.hi.y, b.hi.y); a.hi.z = fmaxf(a.hi.z, b.hi.z);
}
__device__ __forceinline__ NodeBox ld_box(const NodeBox* p) {
    NodeBox b;
    b.lo = __ldcg(&p->lo);
    b.hi = __ldcg(&p->hi);
    return b;
}
__device__ __forceinline__ void st_box(NodeBox* p, const NodeBox& b) {
    __stcg(&p->lo, b.lo);
    __stcg(&p->hi, b.hi);
}

// Leaf boxes (sphere boxes, trbvh.hpp:287), leaf costs, code deltas.
__global__ void k_tr_leaves(uint32_t n, const float4* __restrict__ obj_m, const uint64_t* __restrict__ codes,
                            NodeBox* boxes, float* sah, uint32_t* subtree, uint64_t* delta, uint32_t* touched,
                            bool area3d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = obj_m[i];
    NodeBox b;
    b.lo = make_float4(p.x - p.w, p.y - p.w, p.z - p.w, 0.f);
    b.hi = make_float4(p.x + p.w, p.y + p.w, p.z + p.w, 0.f);
    boxes[i] = b;
    sah[i] = kCt * area_of(b, area3d);
    subtree[i] = 1;
    if (i + 1 < n) {
        delta[i] = codes[i] ^ codes[i + 1];
        touched[i] = 0;
    }
}

// Apetrei agglomerative build (trbvh.hpp:315-389): each leaf climbs; at every
// node the parent side is chosen by comparing code deltas, and the second
// thread to reach a parent finishes it and continues.
__global__ void __launch_bounds__(256) k_apetrei(uint32_t n, const uint64_t* __restrict__ delta, uint32_t* cl,
                                                 uint32_t* cr, uint32_t* rmin, uint32_t* rmax, uint32_t* parent,
                                                 uint32_t* subtree, NodeBox* boxes, float* sah, uint32_t* touched,
                                                 uint32_t* root, bool area3d) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t idx = i, imin = i, imax = i;
    for (uint32_t guard = 0; guard <= n; ++guard) {
        if (imin == 0 && imax == n - 1) {
            parent[idx] = 2 * n;
            root[0] = idx;
            return;
        }
        const bool right_parent = imin == 0 || (imax != n - 1 && delta[imax] < delta[imin - 1]);
        uint32_t p;
        if (right_parent) {
            p = imax + n;
            __stcg(&cl[p - n], idx);
            __stcg(&rmin[p - n], imin);
        } else {
            p = imin + n - 1;
            __stcg(&cr[p - n], idx);
            __stcg(&rmax[p - n], imax);
        }
        __stcg(&parent[idx], p);
        if (atom_add_acq_rel(&touched[p - n], 1u) == 0u) return;
        const uint32_t l = __ldcg(&cl[p - n]), r = __ldcg(&cr[p - n]);
        NodeBox b = ld_box(&boxes[l]);
        box_union(b, ld_box(&boxes[r]));
        st_box(&boxes[p], b);
        __stcg(&subtree[p], __ldcg(&subtree[l]) + __ldcg(&subtree[r]));
        __stcg(&sah[p], (ci_area_of(b, area3d) + __ldcg(&sah[l])) + __ldcg(&sah[r]));
        idx = p;
        if (right_parent) imax = __ldcg(&rmax[p - n]);
        else imin = __ldcg(&rmin[p - n]);
    }
}

// Restructure the treelet rooted at internal node idx (trbvh.hpp:407-618).
template <int K>
__device__ void treelet_opt(uint32_t n, uint32_t idx, bool area3d, uint32_t* cl, uint32_t* cr, uint32_t* parent,
                            uint32_t* subtree, NodeBox* boxes, float* sah) {
    uint32_t inner[K], leaves[K];
    float cost[K];
    inner[0] = idx;
    leaves[0] = __ldcg(&cl[idx - n]);
    leaves[1] = __ldcg(&cr[idx - n]);
    cost[0] = __ldcg(&sah[leaves[0]]);
    cost[1] = __ldcg(&sah[leaves[1]]);
    for (int in = 1; in < K - 1; ++in) {
        int best = -1;
        float bc = -FLT_MAX;
        for (int l = 0; l <= in; ++l)
            if (leaves[l] >= n && (best < 0 || cost[l] > bc)) { bc = cost[l]; best = l; }
        if (best < 0) return;
        const uint32_t bl = leaves[best];
        inner[in] = bl;
        leaves[best] = leaves[in];
        cost[best] = cost[in];
        leaves[in] = __ldcg(&cl[bl - n]);
        cost[in] = __ldcg(&sah[leaves[in]]);
        leaves[in + 1] = __ldcg(&cr[bl - n]);
        cost[in + 1] = __ldcg(&sah[leaves[in + 1]]);
    }
    constexpr int NS = 1 << K, MASK = NS - 1;
    float areas[NS], copt[NS];
    uint8_t popt[NS];
    uint32_t tsz[NS];
    NodeBox lb[K];
    uint32_t lsz[K];
#pragma unroll
    for (int l = 0; l < K; ++l) {
        lb[l] = ld_box(&boxes[leaves[l]]);
        lsz[l] = __ldcg(&subtree[leaves[l]]);
    }
    for (int s = 1; s < NS; ++s) {
        NodeBox b;
        b.lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
        b.hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
        uint32_t sz = 0;
#pragma unroll
        for (int l = 0; l < K; ++l)
            if (s & (1 << l)) { box_union(b, lb[l]); sz += lsz[l]; }
        areas[s] = area_of(b, area3d);
        tsz[s] = sz;
        copt[s] = 0.0f;
        popt[s] = 0;
    }
#pragma unroll
    for (int l = 0; l < K; ++l) copt[1 << l] = cost[l];
    for (int k = 2; k <= K; ++k) {
        for (int s = 1; s < NS; ++s) {
            if (__popc((unsigned)s) != k) continue;
            float cs = FLT_MAX;
            int ps = 0;
            const int dl = (s - 1) & s;
            int p = (-dl) & s;
            while (p != 0) {
                const float c = copt[p] + copt[s ^ p];
                if (c < cs) { cs = c; ps = p; }
                p = (p - dl) & s;
            }
            copt[s] = fminf(kCi * areas[s] + cs, kCt * areas[s] * (float)tsz[s]);
            popt[s] = (uint8_t)ps;
        }
    }
    int index = 0;
    uint8_t stp[2 * K], stl[2 * K];
    uint32_t stpar[2 * K];
    int ss = 0;
    __stcg(&sah[idx], copt[MASK]);
    stp[ss] = popt[MASK]; stl[ss] = 1; stpar[ss] = inner[0]; ++ss;
    stp[ss] = (uint8_t)((~popt[MASK]) & MASK); stl[ss] = 0; stpar[ss] = inner[0]; ++ss;
    while (ss) {
        --ss;
        const int part = stp[ss];
        const bool isl = stl[ss];
        const uint32_t par = stpar[ss];
        const bool leaf = __popc((unsigned)part) == 1;
        const uint32_t node = leaf ? leaves[__ffs(part) - 1] : inner[++index];
        if (isl) __stcg(&cr[par - n], node);
        else __stcg(&cl[par - n], node);
        __stcg(&parent[node], par);
        if (!leaf) {
            NodeBox b;
            b.lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
            b.hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
#pragma unroll
            for (int l = 0; l < K; ++l)
                if (part & (1 << l)) box_union(b, lb[l]);
            st_box(&boxes[node], b);
            __stcg(&subtree[node], tsz[part]);
            __stcg(&sah[node], copt[part]);
            const int pl = popt[part], pr = (~pl) & part;
            stp[ss] = (uint8_t)pl; stl[ss] = 1; stpar[ss] = node; ++ss;
            stp[ss] = (uint8_t)pr; stl[ss] = 0; stpar[ss] = node; ++ss;
        }
    }
}

// Subsets of a K-leaf treelet ordered by size (the DP's levels): subsets of
// size k are list[off[k] .. off[k + 1]).
template <int K>
struct SubsetLevels {
    uint8_t list[(1 << K) - 1];
    uint8_t off[K + 2];
};
template <int K>
constexpr SubsetLevels<K> make_levels() {
    SubsetLevels<K> t{};
    int c = 0;
    for (int k = 1; k <= K; ++k) {
        t.off[k] = (uint8_t)c;
        for (int s = 1; s < (1 << K); ++s) {
            int pc = 0;
            for (int b = 0; b < K; ++b) pc += (s >> b) & 1;
            if (pc == k) t.list[c++] = (uint8_t)s;
        }
    }
    t.off[K + 1] = (uint8_t)c;
    t.off[0] = 0;
    return t;
}
__constant__ SubsetLevels<3> c_lv3 = make_levels<3>();
__constant__ SubsetLevels<4> c_lv4 = make_levels<4>();
__constant__ SubsetLevels<5> c_lv5 = make_levels<5>();
__constant__ SubsetLevels<6> c_lv6 = make_levels<6>();
__constant__ SubsetLevels<7> c_lv7 = make_levels<7>();
__constant__ SubsetLevels<8> c_lv8 = make_levels<8>();
template <int K> __device__ __forceinline__ const SubsetLevels<K>& levels();
template <> __device__ __forceinline__ const SubsetLevels<3>& levels<3>() { return c_lv3; }
template <> __device__ __forceinline__ const SubsetLevels<4>& levels<4>() { return c_lv4; }
template <> __device__ __forceinline__ const SubsetLevels<5>& levels<5>() { return c_lv5; }
template <> __device__ __forceinline__ const SubsetLevels<6>& levels<6>() { return c_lv6; }
template <> __device__ __forceinline__ const SubsetLevels<7>& levels<7>() { return c_lv7; }
template <> __device__ __forceinline__ const SubsetLevels<8>& levels<8>() { return c_lv8; }

// Per-warp scratch of the cooperative treelet DP.
struct TreeletScratch {
    float areas[256], copt[256];
    uint32_t tsz[256];
    uint8_t popt[256];
};

// The treelet rooted at internal node idx restructured by the whole warp
// (trbvh.hpp:407-618): every lane forms the same treelet (reads only), the
// subset areas and each level of the DP are split over the lanes (each
// subset's partitions in the serial order, so every value is the serial
// one), and lane `owner` rebuilds the treelet and writes it.
template <int K>
__device__ void treelet_opt_warp(uint32_t n, uint32_t idx, bool area3d, uint32_t* cl, uint32_t* cr, uint32_t* parent,
                                 uint32_t* subtree, NodeBox* boxes, float* sah, TreeletScratch& W, bool owner) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t inner[K], leaves[K];
    float cost[K];
    inner[0] = idx;
    leaves[0] = __ldcg(&cl[idx - n]);
    leaves[1] = __ldcg(&cr[idx - n]);
    cost[0] = __ldcg(&sah[leaves[0]]);
    cost[1] = __ldcg(&sah[leaves[1]]);
    bool formed = true;
    for (int in = 1; in < K - 1; ++in) {
        int best = -1;
        float bc = -FLT_MAX;
        for (int l = 0; l <= in; ++l)
            if (leaves[l] >= n && (best < 0 || cost[l] > bc)) { bc = cost[l]; best = l; }
        if (best < 0) { formed = false; break; }
        const uint32_t bl = leaves[best];
        inner[in] = bl;
        leaves[best] = leaves[in];
        cost[best] = cost[in];
        leaves[in] = __ldcg(&cl[bl - n]);
        cost[in] = __ldcg(&sah[leaves[in]]);
        leaves[in + 1] = __ldcg(&cr[bl - n]);
        cost[in + 1] = __ldcg(&sah[leaves[in + 1]]);
    }
    if (!formed) return;  // the same on every lane
    constexpr int NS = 1 << K, MASK = NS - 1;
    NodeBox lb[K];
    uint32_t lsz[K];
#pragma unroll
    for (int l = 0; l < K; ++l) {
        lb[l] = ld_box(&boxes[leaves[l]]);
        lsz[l] = __ldcg(&subtree[leaves[l]]);
    }
    for (int s = 1 + (int)lane; s < NS; s += 32) {
        NodeBox b;
        b.lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
        b.hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
        uint32_t sz = 0;
#pragma unroll
        for (int l = 0; l < K; ++l)
            if (s & (1 << l)) { box_union(b, lb[l]); sz += lsz[l]; }
        W.areas[s] = area_of(b, area3d);
        W.tsz[s] = sz;
        W.copt[s] = 0.0f;
        W.popt[s] = 0;
    }
    __syncwarp();
    if (lane < (uint32_t)K) W.copt[1 << lane] = cost[lane];
    __syncwarp();
    const SubsetLevels<K>& LV = levels<K>();
    for (int k = 2; k <= K; ++k) {
        for (int m = LV.off[k] + (int)lane; m < LV.off[k + 1]; m += 32) {
            const int s = LV.list[m];
            float cs = FLT_MAX;
            int ps = 0;
            const int dl = (s - 1) & s;
            int p = (-dl) & s;
            while (p != 0) {
                const float c = W.copt[p] + W.copt[s ^ p];
                if (c < cs) { cs = c; ps = p; }
                p = (p - dl) & s;
            }
            W.copt[s] = fminf(kCi * W.areas[s] + cs, kCt * W.areas[s] * (float)W.tsz[s]);
            W.popt[s] = (uint8_t)ps;
        }
        __syncwarp();
    }
    if (owner) {
        int index = 0;
        uint8_t stp[2 * K], stl[2 * K];
        uint32_t stpar[2 * K];
        int ss = 0;
        __stcg(&sah[idx], W.copt[MASK]);
        stp[ss] = W.popt[MASK]; stl[ss] = 1; stpar[ss] = inner[0]; ++ss;
        stp[ss] = (uint8_t)((~W.popt[MASK]) & MASK); stl[ss] = 0; stpar[ss] = inner[0]; ++ss;
        while (ss) {
            --ss;
            const int part = stp[ss];
            const bool isl = stl[ss];
            const uint32_t par = stpar[ss];
            const bool leaf = __popc((unsigned)part) == 1;
            const uint32_t node = leaf ? leaves[__ffs(part) - 1] : inner[++index];
            if (isl) __stcg(&cr[par - n], node);
            else __stcg(&cl[par - n], node);
            __stcg(&parent[node], par);
            if (!leaf) {
                NodeBox b;
                b.lo = make_float4(FLT_MAX, FLT_MAX, FLT_MAX, 0.f);
                b.hi = make_float4(-FLT_MAX, -FLT_MAX, -FLT_MAX, 0.f);
#pragma unroll
                for (int l = 0; l < K; ++l)
                    if (part & (1 << l)) box_union(b, lb[l]);
                st_box(&boxes[node], b);
                __stcg(&subtree[node], W.tsz[part]);
                __stcg(&sah[node], W.copt[part]);
                const int pl = W.popt[part], pr = (~pl) & part;
                stp[ss] = (uint8_t)pl; stl[ss] = 1; stpar[ss] = node; ++ss;
                stp[ss] = (uint8_t)pr; stl[ss] = 0; stpar[ss] = node; ++ss;
            }
        }
    }
    __syncwarp();
}

// One restructuring round (trbvh.hpp:392-633): leaves climb with the
// second-arrival rule; every internal node whose subtree holds at least
// min_size objects is restructured once, after its whole subtree.  The
// treelets that the lanes of a warp reach are restructured one after the
// other by the whole warp; a lane that has stopped climbing keeps helping.
template <int K>
// 64 registers (16 blocks of 64 per SM): 11.12 ms for the three treelet-7
// rounds at 4M against 11.51 ms at 80 registers and 12.21 ms at 48.
__global__ void __launch_bounds__(64, 16) k_treelets(uint32_t n, uint32_t min_size, bool area3d, uint32_t* cl,
                                                 uint32_t* cr, uint32_t* parent, uint32_t* subtree, NodeBox* boxes,
                                                 float* sah, uint32_t* touched) {
    __shared__ TreeletScratch s_w[2];
    TreeletScratch& W = s_w[threadIdx.x >> 5];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    bool alive = i < n;
    uint32_t idx = i;
    uint32_t par = alive ? __ldcg(&parent[i]) : 0u;
    uint32_t size = 1;
    for (uint32_t guard = 0; guard <= n; ++guard) {
        const bool want = alive && idx >= n && size >= min_size;
        uint32_t m = __ballot_sync(0xffffffffu, want);
        while (m) {
            const uint32_t src = (uint32_t)__ffs(m) - 1u;
            m &= m - 1u;
            const uint32_t root = __shfl_sync(0xffffffffu, idx, src);
            __syncwarp();
            treelet_opt_warp<K>(n, root, area3d, cl, cr, parent, subtree, boxes, sah, W, lane == src);
        }
        if (alive) {
            if (par == 2 * n) {
                alive = false;
            } else if (atom_add_acq_rel(&touched[par - n], 1u) == 0u) {
                alive = false;
            } else {
                idx = par;
                size = __ldcg(&subtree[idx]);
                par = __ldcg(&parent[idx]);
            }
        }
        if (!__any_sync(0xffffffffu, alive)) break;
    }
}

__global__ void __launch_bounds__(128) k_tr_count(uint32_t n, const float4* __restrict__ obj_m,
                                                  const uint32_t* __restrict__ cl, const uint32_t* __restrict__ cr,
                                                  const NodeBox* __restrict__ boxes, const uint32_t* __restrict__ root,
                                                  uint32_t* __restrict__ out) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    uint32_t st[96];
    uint32_t ss = 0, c = 0;
    st[ss++] = root[0];
    const float4 s = obj_m[q];
    while (ss) {
        const uint32_t cur = st[--ss];
        const uint32_t ch[2] = {cl[cur - n], cr[cur - n]};
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const uint32_t x = ch[k];
            if (x >= n) {
                const NodeBox b = boxes[x];
                const bool in = (s.x - s.w < b.hi.x) && (s.x + s.w > b.lo.x) && (s.y - s.w < b.hi.y) &&
                                (s.y + s.w > b.lo.y) && (s.z - s.w < b.hi.z) && (s.z + s.w > b.lo.z);
                if (in && ss < 96) st[ss++] = x;
            } else if (x != q) {
                const float4 o = obj_m[x];
                const float rs = s.w + o.w;
                const float dx = s.x - o.x, dy = s.y - o.y, dz = s.z - o.z;
                if (dx * dx + dy * dy + dz * dz <= rs * rs) ++c;
            }
        }
    }
    out[q] = c;
}

}  // namespace

void TRBVH3D::build(const float4* d_obj, uint32_t n_, cudaStream_t stream, uint32_t* d_status, StageMarks* prof) {
    if (n_ < 2) throw std::invalid_argument("TRBVH3D: needs at least 2 objects");
    if (treelet_size < 3 || treelet_size > kTreeletMax) throw std::invalid_argument("TRBVH3D: treelet size in [3, 8]");
    n = n_;
    sorter.bits = 63;
    sorter.fit_point = false;
    sorter.sort_stage(d_obj, n, stream, d_status, prof);
    if (prof) prof->mark_hierarchy();
    const size_t m = 2 * (size_t)n - 1;
    child_left.ensure(n - 1); child_right.ensure(n - 1); range_min.ensure(n - 1); range_max.ensure(n - 1);
    parent.ensure(m); subtree_size.ensure(m); boxes.ensure(m); sah.ensure(m);
    delta.ensure(n - 1); touched.ensure(n - 1); root.ensure(1);
    k_tr_leaves<<<grid_for(n, 256), 256, 0, stream>>>(n, sorter.obj_m.ptr, sorter.codes.ptr, boxes.ptr, sah.ptr,
                                                      subtree_size.ptr, delta.ptr, touched.ptr, area3d);
    SB_LAUNCH_CHECK();
    k_apetrei<<<grid_for(n, 256), 256, 0, stream>>>(n, delta.ptr, child_left.ptr, child_right.ptr, range_min.ptr,
                                                    range_max.ptr, parent.ptr, subtree_size.ptr, boxes.ptr, sah.ptr,
                                                    touched.ptr, root.ptr, area3d);
    SB_LAUNCH_CHECK();
    if (prof) prof->mark_treelets();
    uint32_t min_size = (uint32_t)treelet_size;
    for (int r = 0; r < rounds; ++r) {
        SB_CUDA(cudaMemsetAsync(touched.ptr, 0, sizeof(uint32_t) * (n - 1), stream));
#define SB_TREELET(K)                                                                                           \
    k_treelets<K><<<grid_for(n, 64), 64, 0, stream>>>(n, min_size, area3d, child_left.ptr, child_right.ptr,  \
                                                       parent.ptr, subtree_size.ptr, boxes.ptr, sah.ptr, touched.ptr)
        switch (treelet_size) {
            case 3: SB_TREELET(3); break;
            case 4: SB_TREELET(4); break;
            case 5: SB_TREELET(5); break;
            case 6: SB_TREELET(6); break;
            case 7: SB_TREELET(7); break;
            default: SB_TREELET(8); break;
        }
#undef SB_TREELET
        SB_LAUNCH_CHECK();
        min_size *= 2;
    }
}

void TRBVH3D::count_overlaps(uint32_t* d_out, cudaStream_t stream) const {
    k_tr_count<<<grid_for(n, 128), 128, 0, stream>>>(n, sorter.obj_m.ptr, child_left.ptr, child_right.ptr, boxes.ptr,
                                                     root.ptr, d_out);
    SB_LAUNCH_CHECK();
}

}  // namespace sb
