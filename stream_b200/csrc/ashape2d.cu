// 2D direct alpha shape kernels for sm_100a (compiled with -fmad=false so the
// reference's non-exact float tests are evaluated as separate IEEE operations;
// the explicit fmaf() calls of its in-circle filter stay fused).
#include <algorithm>
#include <cstring>

#include "ashape2d.cuh"
#include "predicates.cuh"

namespace sb {
namespace {

// 2*delta, delta = sqrt((1+4eps)/(1-3eps)) (DirectAlphaShape2D.cpp:185-188, 318-320).
constexpr float kTwoDelta2 = 2.0000004172325445139859201780136934301654f;
constexpr int kStar2Block = 64;

__global__ void k_pack_nodes2d(uint32_t n, const float* __restrict__ coords, const float* __restrict__ alpha,
                               float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_float4(coords[2 * (size_t)i], coords[2 * (size_t)i + 1], 0.0f, alpha[i]);
}

// Infinity points around the global box (DirectAlphaShape2D.cpp:144-166):
// bottom left, bottom right, top; radius 0.  bb = pmin[3], pmax[3].
__global__ void k_infinity2d(const float* bb, float4* cm, uint32_t n) {
    if (threadIdx.x != 0) return;
    const float avg0 = 0.5f * (bb[3] + bb[0]), avg1 = 0.5f * (bb[4] + bb[1]);
    const float mr = fmaxf(bb[3] - bb[0], bb[4] - bb[1]);
    const float two = 2.0f * mr;
    cm[n + 0] = make_float4(avg0 - two, avg1 - two, 0.0f, 0.0f);
    cm[n + 1] = make_float4(avg0 + two, avg1 - two, 0.0f, 0.0f);
    cm[n + 2] = make_float4(avg0, avg1 + two, 0.0f, 0.0f);
}

// Disk-box test of the neighbour search (:202-209, :335-342).
__device__ __forceinline__ bool disk_hits(const float4 si, float rs2, const NodeBox& b) {
    const float dmaxx = fmaxf(si.x - b.hi.x, 0.0f);
    const float dmaxy = fmaxf(si.y - b.hi.y, 0.0f);
    const float dminx = fmaxf(b.lo.x - si.x, 0.0f);
    const float dminy = fmaxf(b.lo.y - si.y, 0.0f);
    return dmaxx * dmaxx + dminx * dminx + dmaxy * dmaxy + dminy * dminy < rs2;
}
// Neighbour predicate ||si - sj||^2 < (2 delta min(alpha_i, alpha_j))^2 (:211-218, :343-349).
__device__ __forceinline__ bool near2(const float4 si, const float4 sj) {
    const float ma = fminf(si.w, sj.w);
    const float dx = si.x - sj.x, dy = si.y - sj.y;
    const float lim = (kTwoDelta2 * ma) * (kTwoDelta2 * ma);
    return dx * dx + dy * dy < lim;
}

__device__ __forceinline__ NodeBox load_box(const NodeBox* boxes, uint32_t c) {
    NodeBox b;
    b.lo = __ldg(&boxes[c].lo);
    b.hi = __ldg(&boxes[c].hi);
    return b;
}

// Count pass (:178-224): neighbours of each point (self excluded), and per
// warp block of 32 points 32 x its largest count (the ELL block size, :254-266).
// The count does not depend on the visiting order, so the search continues
// with one intersecting child directly and pushes only the other.
__global__ void __launch_bounds__(128) k_count2d(const float4* __restrict__ cm, uint32_t n,
                                                 const int32_t* __restrict__ sep, const uint8_t* __restrict__ cil,
                                                 const NodeBox* __restrict__ boxes, uint32_t* __restrict__ bsz,
                                                 uint32_t* words) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t k = 0;
    bool overflow = false;
    if (tid < n) {
        int stack[64];
        int ss = 0, cur = 0;
        const float4 si = cm[tid];
        const float rs = kTwoDelta2 * si.w;
        const float rs2 = rs * rs;
        for (;;) {
            if (cur < 0) {
                if (ss == 0) break;
                cur = stack[--ss];
            }
            const uint32_t s = (uint32_t)__ldg(&sep[cur]);
            const uint8_t cl = __ldg(&cil[cur]);
            cur = -1;
#pragma unroll
            for (uint32_t ch = 0; ch < 2; ++ch) {
                const uint32_t c = s + ch;
                if (!(cl & (ch + 1))) {
                    if (disk_hits(si, rs2, load_box(boxes, c))) {
                        if (cur >= 0) {
                            if (ss < 64) stack[ss++] = cur;
                            else overflow = true;
                        }
                        cur = (int)c;
                    }
                } else if (c != tid && near2(si, __ldg(&cm[c]))) {
                    ++k;
                }
            }
        }
    }
    const uint32_t m = __reduce_max_sync(0xffffffffu, k);
    // the fill pass stops at kFillLimit2 + 2 local ids at most
    if ((threadIdx.x & 31) == 0 && tid < n) bsz[tid >> 5] = 32u * min(m + kInf2, kFillLimit2 + 2);
    if (overflow) atomicOr(&words[0], ST_STACK_OVERFLOW);
}

// Fill pass (:310-357) in the reference's visiting order: the children of a
// popped node are tested child 0 then child 1, intersecting internal children
// pushed in that order.  Stops after the node at which the star holds more
// than kFillLimit2 local ids.
__global__ void __launch_bounds__(128) k_fill2d(const float4* __restrict__ cm, uint32_t n,
                                                const int32_t* __restrict__ sep, const uint8_t* __restrict__ cil,
                                                const NodeBox* __restrict__ boxes, const uint32_t* __restrict__ boff,
                                                uint32_t* __restrict__ cand, float2* __restrict__ ccoord,
                                                uint32_t* __restrict__ nineig, uint32_t* words) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= n) return;
    const size_t off = (size_t)boff[tid >> 5] + (tid & 31);
    const uint32_t cap = (boff[(tid >> 5) + 1] - boff[tid >> 5]) >> 5;  // local ids incl. infinity
#pragma unroll
    for (uint32_t q = 0; q < kInf2; ++q) {
        const float4 v = cm[n + q];
        cand[off + 32 * q] = n + q;
        ccoord[off + 32 * q] = make_float2(v.x, v.y);
    }
    int stack[64];
    int ss = 0, cur = 0;
    const float4 si = cm[tid];
    const float rs = kTwoDelta2 * si.w;
    const float rs2 = rs * rs;
    uint32_t k = kInf2;
    bool overflow = false, limited = false;
    for (;;) {
        if (cur < 0) {
            if (ss == 0) break;
            cur = stack[--ss];
        }
        const uint32_t s = (uint32_t)__ldg(&sep[cur]);
        const uint8_t cl = __ldg(&cil[cur]);
        cur = -1;
#pragma unroll
        for (uint32_t ch = 0; ch < 2; ++ch) {
            const uint32_t c = s + ch;
            if (!(cl & (ch + 1))) {
                if (disk_hits(si, rs2, load_box(boxes, c))) {
                    if (cur >= 0) {  // child 0 goes below child 1 on the stack
                        if (ss < 64) stack[ss++] = cur;
                        else overflow = true;
                    }
                    cur = (int)c;
                }
            } else if (c != tid) {
                const float4 sj = __ldg(&cm[c]);
                if (near2(si, sj)) {
                    const uint32_t j = k;  // local id
                    if (j < cap) {
                        cand[off + 32 * (size_t)j] = c;
                        ccoord[off + 32 * (size_t)j] = make_float2(sj.x, sj.y);
                    } else {
                        overflow = true;
                    }
                    ++k;
                }
            }
        }
        if (k > kFillLimit2) {
            limited = true;
            break;
        }
    }
    nineig[tid] = k;
    if (limited) atomicAdd(&words[1], 1u);
    if (overflow) atomicOr(&words[0], ST_STACK_OVERFLOW);
}

struct Star2Params {
    uint32_t n;
    const float4* cm;
    const uint32_t* boff;
    const uint32_t* cand;
    const float2* ccoord;
    const uint32_t* nineig;
    uint32_t* tris;
    uint8_t* act;
    uint32_t* nout;
    uint32_t* nfneig;
    uint8_t* nkeep;
    uint8_t* node_is_bnd;
    uint32_t* words;
};

// One star (:373-600): insertion loop with swap-with-last deletion of the
// conflicting triangles, their vertices toggled in a 256-bit parity set
// (thread-private words in shared memory, stride kStar2Block); the set bits
// (the cavity boundary) become new triangles (r, ni) in increasing r.  Then
// infinity removal, alpha filter, orientation and the owner count.
__device__ void star2_one(const Star2Params& P, uint32_t si, unsigned long long (*par)[kStar2Block]) {
    const uint32_t t = threadIdx.x;
    const uint32_t w = si >> 5;
    const size_t coff = (size_t)P.boff[w] + (si & 31);
    const uint32_t tcap = (P.boff[w + 1] - P.boff[w]) >> 5;  // neighbours + 3 >= triangles of the star
    uint32_t* T = P.tris + coff;
    const float2* C = P.ccoord + coff;  // local id a at C[32 a] (0..2: infinity points)
    const uint32_t* G = P.cand + coff;
    const uint32_t k = P.nineig[si];
    if (k - kInf2 < 2) {
        P.node_is_bnd[si] = 1;
        P.nout[si] = 0;
        P.nkeep[si] = 0;
        P.nfneig[si] = 0;
        return;
    }
    const float4 c4 = P.cm[si];
    const float2 pa = make_float2(c4.x, c4.y);
    auto coord = [&](uint32_t a) -> float2 { return C[32 * a]; };
    auto gid = [&](uint32_t a) -> uint32_t { return G[32 * a]; };
    uint32_t st = 0, nex = 0;
    // Local triangles (si, a, b) as a | b << 8 | neg << 16, neg = orient2d(si, a, b) < 0:
    // a triangle's orientation is fixed, so it is evaluated once, when the
    // triangle is made, instead of at every in-circle test.
    auto make_tri = [&](uint32_t a, uint32_t b, float2 pb, float2 pc) -> uint32_t {
        return a | (b << 8) | (pred::orient2d(pa, pb, pc, st) < 0.0f ? 1u << 16 : 0u);
    };
    T[0] = make_tri(1, 2, C[32], C[64]);
    T[32] = make_tri(2, 0, C[64], C[0]);
    T[64] = make_tri(0, 1, C[0], C[32]);
    uint32_t Tl = 3;
    for (uint32_t ni = kInf2; ni < k; ++ni) {
        par[0][t] = 0ull;
        par[1][t] = 0ull;
        par[2][t] = 0ull;
        par[3][t] = 0ull;
        const float2 pd = C[32 * ni];
        uint32_t R = 0, ti = 0;
        while (ti < Tl) {
            const uint32_t tr = T[32 * (size_t)ti];
            const uint32_t a = tr & 255u, b = (tr >> 8) & 255u;
            const float2 pb = coord(a), pc = coord(b);
            const float orientation = (tr >> 16) ? -1.0f : 1.0f;  // only its sign is used
            float err;
            float det = pred::incircle32(pa, pb, pc, pd, err);
            if (!((det > err) || (-det > err))) {
                ++nex;
                det = pred::incircle_sos(pa, pb, pc, pd, si, gid(a), gid(b), gid(ni), orientation, st);
            }
            if (orientation < 0.0f) det = -det;
            if (det > 0.0f) {
                par[a >> 6][t] ^= 1ull << (a & 63);
                par[b >> 6][t] ^= 1ull << (b & 63);
                ++R;
                --Tl;
                T[32 * (size_t)ti] = T[32 * (size_t)Tl];
            } else {
                ++ti;
            }
        }
        if (R) {
            for (uint32_t j = 0; j < 4; ++j) {
                unsigned long long v = par[j][t];
                while (v) {  // set bits in increasing order; all are below ni
                    const uint32_t r = 64 * j + (uint32_t)(__ffsll((long long)v) - 1);
                    v &= v - 1;
                    if (Tl < tcap) T[32 * (size_t)Tl++] = make_tri(r, ni, coord(r), pd);
                    else st |= ST_TET_CAP;
                }
            }
        }
    }
    // ---- filter (:528-595) ----
    bool bnd = false;
    uint32_t nout = 0, nkeep = 0, nf = 0;
    uint32_t ti = 0;
    while (ti < Tl) {
        const uint32_t tr = T[32 * (size_t)ti];
        const uint32_t a = tr & 255u, b = (tr >> 8) & 255u;
        if (a < kInf2 || b < kInf2) {
            bnd = true;
            --Tl;
            T[32 * (size_t)ti] = T[32 * (size_t)Tl];
            continue;
        }
        uint32_t i1 = si, i2 = gid(a), i3 = gid(b), tmp;
        bool swp = false;
        if (i3 < i2) { tmp = i3; i3 = i2; i2 = tmp; swp = !swp; }
        if (i2 < i1) { tmp = i2; i2 = i1; i1 = tmp; swp = !swp; }
        if (i3 < i2) { tmp = i3; i3 = i2; i2 = tmp; swp = !swp; }
        const float4 p1 = __ldg(&P.cm[i1]), p2 = __ldg(&P.cm[i2]), p3 = __ldg(&P.cm[i3]);
        float det = (p3.x - p2.x) * (p1.y - p2.y) - (p3.y - p2.y) * (p1.x - p2.x);
        if (swp) det = -det;
        const float ax = p1.x - p2.x, ay = p1.y - p2.y;
        const float bx = p2.x - p3.x, by = p2.y - p3.y;
        const float cx = p3.x - p1.x, cy = p3.y - p1.y;
        const float l12 = ax * ax + ay * ay, l23 = bx * bx + by * by, l31 = cx * cx + cy * cy;
        const float crs = (l12 * l23 * l31) / (4.f * det * det);
        const float aeff = fminf(p3.w, fminf(p1.w, p2.w));
        if (crs <= aeff * aeff) {
            uint8_t* pa8 = P.act + coff + 32 * (size_t)a;
            uint8_t* pb8 = P.act + coff + 32 * (size_t)b;
            const uint8_t ca = *pa8, cb = *pb8;
            nf += (ca == 0) + (cb == 0);
            *pa8 = (uint8_t)(ca + 1);
            *pb8 = (uint8_t)(cb + 1);
            ++nkeep;
            if (det < 0.0f) T[32 * (size_t)ti] = b | (a << 8);
            ++ti;
            nout += (si == i1);
        } else {
            bnd = true;
            --Tl;
            T[32 * (size_t)ti] = T[32 * (size_t)Tl];
        }
    }
    P.node_is_bnd[si] = bnd ? 1 : 0;
    P.nout[si] = nout;
    P.nkeep[si] = (uint8_t)nkeep;
    P.nfneig[si] = nf;
    if (st) atomicOr(&P.words[0], st);
    if (nex) atomicAdd(&P.words[2], nex);
}

// Persistent: each lane takes the next star (words[6]) when it finishes one,
// instead of idling until the longest star of its warp is done.
__global__ void __launch_bounds__(kStar2Block) k_star2d(Star2Params P) {
    __shared__ unsigned long long par[4][kStar2Block];
    for (;;) {
        const uint32_t si = atomicAdd(&P.words[6], 1u);
        if (si >= P.n) break;
        star2_one(P, si, par);
    }
}

// Compress (:642-690): CSR edges with boundary flags, and the triangles this
// point owns (it is their smallest id) in local order.
__global__ void __launch_bounds__(128) k_compress2d(uint32_t n, const uint32_t* __restrict__ boff,
                                                    const uint32_t* __restrict__ cand,
                                                    const uint32_t* __restrict__ tris,
                                                    const uint8_t* __restrict__ act,
                                                    const uint32_t* __restrict__ nineig,
                                                    const uint32_t* __restrict__ row,
                                                    const uint32_t* __restrict__ elemrow, uint32_t* __restrict__ neig,
                                                    uint8_t* __restrict__ edge_is_bnd, uint32_t* __restrict__ elems) {
    const uint32_t si = blockIdx.x * blockDim.x + threadIdx.x;
    if (si >= n) return;
    const uint32_t w = si >> 5;
    const size_t coff = (size_t)boff[w] + (si & 31);
    const uint32_t* T = tris + coff;
    uint32_t put = row[si];
    const uint32_t k = nineig[si];
    for (uint32_t i = kInf2; i < k; ++i) {
        const uint8_t c = act[coff + 32 * (size_t)i];
        if (c) {
            edge_is_bnd[put] = (c == 1);
            neig[put++] = cand[coff + 32 * (size_t)i];
        }
    }
    auto gid = [&](uint32_t a) -> uint32_t { return cand[coff + 32 * (size_t)a]; };
    uint32_t idx = 0;
    const uint32_t e1 = elemrow[si + 1];
    for (uint32_t i = elemrow[si]; i < e1; ++i) {
        uint32_t tr = T[32 * (size_t)idx];
        uint32_t a = gid(tr & 255u), b = gid((tr >> 8) & 255u);
        while (a < si || b < si) {
            ++idx;
            tr = T[32 * (size_t)idx];
            a = gid(tr & 255u);
            b = gid((tr >> 8) & 255u);
        }
        elems[3 * (size_t)i] = si;
        elems[3 * (size_t)i + 1] = a;
        elems[3 * (size_t)i + 2] = b;
        ++idx;
    }
}

}  // namespace

AlphaShape2D::AlphaShape2D() {
    SB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
    lbvh.fit_point = true;
    lbvh.tail = kInf2;
    lbvh.bits = 64;
    words.ensure(8);
}

AlphaShape2D::~AlphaShape2D() {
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
    if (own_stream_saved) cudaStreamDestroy(own_stream_saved);
}

void AlphaShape2D::set_stream(cudaStream_t s) {
    SB_CUDA(cudaStreamSynchronize(stream));
    if (s) {
        if (own_stream) own_stream_saved = stream;
        stream = s;
        own_stream = false;
    } else if (own_stream_saved) {
        stream = own_stream_saved;
        own_stream_saved = nullptr;
        own_stream = true;
    }
}

void AlphaShape2D::mark(int i) {
    if (!profiling) return;
    if (!ev[i]) SB_CUDA(cudaEventCreate(&ev[i]));
    SB_CUDA(cudaEventRecord(ev[i], stream));
}

void AlphaShape2D::collect_profile() {
    if (!profiling) return;
    SB_CUDA(cudaEventSynchronize(ev[S_COUNT]));
    for (int i = 0; i < S_COUNT; ++i) {
        float ms = 0.f;
        SB_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
        stage_ms[i] = ms;
    }
}

// Largest point count: the lane-interleaved slots (<= 252 local ids per point)
// must stay below 2^32.
constexpr uint32_t kMaxNodes2D = 16u * 1024u * 1024u;

void AlphaShape2D::set_nodes_host(uint32_t n, const float* coords, const float* alpha) {
    if (n < 2 || n > kMaxNodes2D) throw std::invalid_argument("AlphaShape2D needs 2 to 16M nodes");
    staging.ensure((size_t)3 * n);
    SB_CUDA(cudaMemcpyAsync(staging.ptr, coords, sizeof(float) * 2 * (size_t)n, cudaMemcpyHostToDevice, stream));
    SB_CUDA(cudaMemcpyAsync(staging.ptr + 2 * (size_t)n, alpha, sizeof(float) * n, cudaMemcpyHostToDevice, stream));
    input_bad.ensure(1);
    if (any_nonfinite(staging.ptr, (size_t)3 * n, input_bad.ptr, pinned.h + 12, stream)) {  // before any meshing kernel
        n_nodes = 0;
        inited = computed = false;
        throw std::invalid_argument("AlphaShape2D::set_nodes: a coordinate or an alpha is infinite or NaN");
    }
    nodes.ensure(n);
    k_pack_nodes2d<<<grid_for(n, 256), 256, 0, stream>>>(n, staging.ptr, staging.ptr + 2 * (size_t)n, nodes.ptr);
    SB_LAUNCH_CHECK();
    n_nodes = n;
    inited = computed = false;
}

void AlphaShape2D::set_nodes_device(uint32_t n, const float4* pts) {
    if (n < 2 || n > kMaxNodes2D) throw std::invalid_argument("AlphaShape2D needs 2 to 16M nodes");
    nodes.ensure(n);
    SB_CUDA(cudaMemcpyAsync(nodes.ptr, pts, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
    n_nodes = n;
    inited = computed = false;
}

void AlphaShape2D::init() {
    if (n_nodes < 2) throw std::invalid_argument("AlphaShape2D::init before set_nodes");
    const uint32_t n = n_nodes;
    const uint32_t W = (n + 31) / 32;
    SB_CUDA(cudaMemsetAsync(words.ptr, 0, 8 * sizeof(uint32_t), stream));
    mark(S_LBVH);
    lbvh.build(nodes.ptr, n, stream, words.ptr, nullptr);
    k_infinity2d<<<1, 32, 0, stream>>>(lbvh.bb_glob.ptr, lbvh.obj_m.ptr, n);
    SB_LAUNCH_CHECK();
    mark(S_COUNT_PASS);
    bsz.ensure(W);
    boff.ensure((size_t)W + 1);
    k_count2d<<<grid_for(n, 128), 128, 0, stream>>>(lbvh.obj_m.ptr, n, lbvh.sep.ptr, lbvh.cil.ptr, lbvh.boxes.ptr,
                                                    bsz.ptr, words.ptr);
    SB_LAUNCH_CHECK();
    exclusive_scan_u32(scan, bsz.ptr, boff.ptr, W, stream);
    SB_CUDA(cudaMemcpyAsync(pinned.h, boff.ptr + W, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    slots = pinned.h[0];
    cand.ensure(slots);
    ccoord.ensure(slots);
    act.ensure(slots);
    tris.ensure(slots);
    inited = true;
    computed = false;
}

void AlphaShape2D::compute() {
    if (!inited) init();
    const uint32_t n = n_nodes;
    nineig.ensure(n);
    nout.ensure(n);
    nfneig.ensure(n);
    nkeep.ensure(n);
    node_is_bnd.ensure(n);
    elemrow.ensure((size_t)n + 1);
    row.ensure((size_t)n + 1);
    mark(S_FILL);
    k_fill2d<<<grid_for(n, 128), 128, 0, stream>>>(lbvh.obj_m.ptr, n, lbvh.sep.ptr, lbvh.cil.ptr, lbvh.boxes.ptr,
                                                   boff.ptr, cand.ptr, ccoord.ptr, nineig.ptr, words.ptr);
    SB_LAUNCH_CHECK();
    if (slots) SB_CUDA(cudaMemsetAsync(act.ptr, 0, slots, stream));
    SB_CUDA(cudaMemsetAsync(words.ptr + 6, 0, sizeof(uint32_t), stream));  // star queue
    mark(S_STAR);
    Star2Params P{n, lbvh.obj_m.ptr, boff.ptr, cand.ptr, ccoord.ptr, nineig.ptr, tris.ptr, act.ptr,
                  nout.ptr, nfneig.ptr, nkeep.ptr, node_is_bnd.ptr, words.ptr};
    k_star2d<<<std::min(grid_for(n, kStar2Block), kNumSMs * 10), kStar2Block, 0, stream>>>(P);  // 10 blocks/SM at 96 registers
    SB_LAUNCH_CHECK();
    mark(S_SCAN);
    exclusive_scan_u32(scan, nout.ptr, elemrow.ptr, n, stream);
    exclusive_scan_u32(scan, nfneig.ptr, row.ptr, n, stream);
    SB_CUDA(cudaMemcpyAsync(pinned.h, elemrow.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaMemcpyAsync(pinned.h + 1, row.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    n_elems = pinned.h[0];
    n_edges = pinned.h[1];
    elems.ensure(3 * (size_t)n_elems);
    neig.ensure(n_edges);
    edge_is_bnd.ensure(n_edges);
    mark(S_COMPRESS);
    k_compress2d<<<grid_for(n, 128), 128, 0, stream>>>(n, boff.ptr, cand.ptr, tris.ptr, act.ptr, nineig.ptr, row.ptr,
                                                       elemrow.ptr, neig.ptr, edge_is_bnd.ptr, elems.ptr);
    SB_LAUNCH_CHECK();
    mark(S_COUNT);
    computed = true;
}

void AlphaShape2D::read_counters() {
    SB_CUDA(cudaMemcpyAsync(pinned.h + 8, words.ptr, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    last_status = pinned.h[8];
    last_limited = pinned.h[9];
    last_exact = pinned.h[10];
}

}  // namespace sb
