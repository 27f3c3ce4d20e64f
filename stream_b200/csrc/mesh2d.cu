// 2D Delaunay triangulation kernels for sm_100a (compiled with -fmad=false:
// the in-circle filter shared with the 2D alpha shape keeps its explicit
// fmaf() calls and nothing else is contracted).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

#include "mesh2d.cuh"
#include "predicates.cuh"

namespace sb {
namespace {

constexpr int kM2Block = 64;
constexpr uint32_t kVerified = 1u << 17;
constexpr uint32_t kNone = 0xffffffffu;
// Queries per star and sweep before the star gives up (status ST_WALK_CAP):
// every query either verifies a triangle or inserts a point, and a star holds
// at most kLocal2 ids and kLocal2 triangles.
constexpr uint32_t kMaxQueries = 4 * kLocal2;
// A triangle too thin for a bounded circle (coincident or collinear points)
// is checked against every point; such a query tests at most kMaxFlatLeaves
// points and gives up (kGiveUp), and its star stops.
constexpr uint32_t kMaxFlatLeaves = 8192;
constexpr uint32_t kGiveUp = 0xfffffffeu;
// LBVH nodes one star may visit in one sweep (a star of a uniform cloud
// visits about a thousand): past it the query gives up and the star stops,
// so that no input makes a sweep run away (runs of equal Morton codes, from
// coincident points, make the LBVH a deep chain).
constexpr uint32_t kMaxVisits = 1u << 16;

__global__ void k_pack_points2d(uint32_t n, const float* __restrict__ xy, float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_float4(xy[2 * (size_t)i], xy[2 * (size_t)i + 1], 0.0f, 0.0f);
}

// Super nodes around the global box (mesh.cpp:92-105): avg -+ (max extent + 10).
__global__ void k_super2d(const float* bb, float4* cm, uint32_t n) {
    if (threadIdx.x != 0) return;
    const float avg0 = 0.5f * (bb[3] + bb[0]), avg1 = 0.5f * (bb[4] + bb[1]);
    const float mr = fmaxf(bb[3] - bb[0], bb[4] - bb[1]) + 10.0f;
    cm[n + 0] = make_float4(avg0 - mr, avg1 - mr, 0.0f, 0.0f);
    cm[n + 1] = make_float4(avg0 + mr, avg1 - mr, 0.0f, 0.0f);
    cm[n + 2] = make_float4(avg0, avg1 + mr, 0.0f, 0.0f);
}

__device__ __forceinline__ float2 xy2(const float4 v) { return make_float2(v.x, v.y); }

// One point's star: local ids (global ids in loc), triangles (p, a, b) in tri.
struct Star {
    uint32_t i, n;
    float2 p;
    uint32_t* G;  // stride 32
    uint32_t* T;  // stride 32
    const float4* cm;
    uint32_t L, Tl, st;

    __device__ uint32_t gid(uint32_t a) const { return G[32 * (size_t)a]; }
    __device__ float2 coord(uint32_t a) const { return xy2(__ldg(&cm[gid(a)])); }
    __device__ uint32_t make_tri(uint32_t a, uint32_t b, float2 pa, float2 pb) {
        return a | (b << 8) | (pred::orient2d(p, pa, pb, st) < 0.0f ? 1u << 16 : 0u);
    }
    // In-circle decision of the 2D star kernel (DirectAlphaShape2D.cpp:437-479):
    // true when point q (global id gq) is strictly inside the circle of
    // triangle tr, with the same filter, exact stage and Simulation of
    // Simplicity for every star.
    __device__ bool conflict(uint32_t tr, float2 q, uint32_t gq) {
        const uint32_t a = tr & 255u, b = (tr >> 8) & 255u;
        const float2 pb = coord(a), pc = coord(b);
        const float orientation = (tr >> 16) & 1u ? -1.0f : 1.0f;
        float err;
        float det = pred::incircle32(p, pb, pc, q, err);
        if (!((det > err) || (-det > err))) det = pred::incircle_sos(p, pb, pc, q, i, gid(a), gid(b), gq, orientation, st);
        if (orientation < 0.0f) det = -det;
        return det > 0.0f;
    }
    // Bowyer-Watson step on the star: the conflicting triangles leave by
    // swap-with-last, their vertices are toggled in a parity set (the two that
    // stay set bound the cavity) and become new triangles with the new point.
    __device__ bool insert(uint32_t gq) {
        if (L >= kLocal2) {
            st |= ST_TET_CAP;
            return false;
        }
        const uint32_t ni = L;
        G[32 * (size_t)ni] = gq;
        ++L;
        const float2 q = xy2(__ldg(&cm[gq]));
        unsigned long long par0 = 0ull, par1 = 0ull;
        uint32_t R = 0, ti = 0;
        while (ti < Tl) {
            const uint32_t tr = T[32 * (size_t)ti];
            if (conflict(tr, q, gq)) {
                const uint32_t a = tr & 255u, b = (tr >> 8) & 255u;
                if (a < 64) par0 ^= 1ull << a; else par1 ^= 1ull << (a - 64);
                if (b < 64) par0 ^= 1ull << b; else par1 ^= 1ull << (b - 64);
                ++R;
                --Tl;
                T[32 * (size_t)ti] = T[32 * (size_t)Tl];
            } else {
                ++ti;
            }
        }
        for (int w = 0; w < 2; ++w) {
            unsigned long long v = w ? par1 : par0;
            while (v) {
                const uint32_t r = 64 * w + (uint32_t)(__ffsll((long long)v) - 1);
                v &= v - 1;
                if (Tl < kLocal2) T[32 * (size_t)Tl++] = make_tri(r, ni, coord(r), q);
                else st |= ST_TET_CAP;
            }
        }
        return R > 0;
    }
};

__device__ __forceinline__ Star load_star(uint32_t i, uint32_t n, const float4* cm, uint32_t* loc, uint32_t* tri,
                                          uint32_t L, uint32_t Tl) {
    const size_t base = (size_t)(i >> 5) * 32 * kLocal2 + (i & 31);
    Star s{i, n, xy2(__ldg(&cm[i])), loc + base, tri + base, cm, L, Tl, 0u};
    return s;
}

// init: each star starts as the fan of the three super triangles around its
// point (the point lies inside the super triangle).
__global__ void k_m2_init(uint32_t n, const float4* __restrict__ cm, uint32_t* loc, uint32_t* tri, uint32_t* nloc,
                          uint32_t* ntri, uint8_t* done, uint32_t* words) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Star s = load_star(i, n, cm, loc, tri, kSuper2, 0);
    for (uint32_t q = 0; q < kSuper2; ++q) s.G[32 * q] = n + q;
    const float2 s0 = xy2(cm[n]), s1 = xy2(cm[n + 1]), s2 = xy2(cm[n + 2]);
    s.T[0] = s.make_tri(1, 2, s1, s2);
    s.T[32] = s.make_tri(2, 0, s2, s0);
    s.T[64] = s.make_tri(0, 1, s0, s1);
    nloc[i] = kSuper2;
    ntri[i] = 3;
    done[i] = 0;
    if (s.st) atomicOr(&words[0], s.st);
}

// insert_morton_neighbors: the kMortonSeed points on each side in Morton
// order, nearest first.
__global__ void __launch_bounds__(kM2Block) k_m2_morton(uint32_t n, const float4* __restrict__ cm, uint32_t* loc,
                                                        uint32_t* tri, uint32_t* nloc, uint32_t* ntri, uint32_t* words) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Star s = load_star(i, n, cm, loc, tri, nloc[i], ntri[i]);
    for (uint32_t d = 1; d <= kMortonSeed; ++d) {
        if (i >= d) s.insert(i - d);
        if (i + d < n) s.insert(i + d);
    }
    nloc[i] = s.L;
    ntri[i] = s.Tl;
    if (s.st) atomicOr(&words[0], s.st);
}

// A point strictly inside the circle of star triangle tr (by the star's
// predicate), other than its three vertices, or kNone.  The circle's centre
// and radius are computed in FP64 (the coordinate differences and their
// products are exact there) and widened by a relative 2^-20; for a triangle
// so thin that this could miss (|cross| below 2^-30 |u| |v|) every box is
// visited, up to kMaxFlatLeaves points.  Every node visited spends one of the
// star's `visits`; kGiveUp when either runs out.  Children are visited
// nearest the star's point first, so the points found tend to be its
// neighbours.
__device__ uint32_t find_intruder(Star& s, uint32_t tr, const int32_t* __restrict__ sep,
                                  const uint8_t* __restrict__ cil, const NodeBox* __restrict__ boxes,
                                  uint32_t& visits) {
    const uint32_t a = tr & 255u, b = (tr >> 8) & 255u;
    const uint32_t ga = s.gid(a), gb = s.gid(b);
    const float2 pa = s.coord(a), pb = s.coord(b);
    const double ux = (double)pa.x - s.p.x, uy = (double)pa.y - s.p.y;
    const double vx = (double)pb.x - s.p.x, vy = (double)pb.y - s.p.y;
    const double cr = ux * vy - uy * vx, uu = ux * ux + uy * uy, vv = vx * vx + vy * vy;
    bool all = !(fabs(cr) > 0x1p-30 * sqrt(uu * vv));
    double cx = 0.0, cy = 0.0, r2 = 0.0;
    if (!all) {
        const double ox = (vy * uu - uy * vv) / (2.0 * cr), oy = (ux * vv - vx * uu) / (2.0 * cr);
        cx = s.p.x + ox;
        cy = s.p.y + oy;
        const double r = sqrt(ox * ox + oy * oy) * (1.0 + 0x1p-20);
        r2 = r * r;
        all = !isfinite(r2);
    }
    auto hits = [&](const float4 lo, const float4 hi) -> bool {
        if (all) return true;
        const double dx = fmax(fmax((double)lo.x - cx, cx - (double)hi.x), 0.0);
        const double dy = fmax(fmax((double)lo.y - cy, cy - (double)hi.y), 0.0);
        return dx * dx + dy * dy <= r2;
    };
    auto dist_p = [&](const float4 lo, const float4 hi) -> float {
        const float dx = fmaxf(fmaxf(lo.x - s.p.x, s.p.x - hi.x), 0.0f);
        const float dy = fmaxf(fmaxf(lo.y - s.p.y, s.p.y - hi.y), 0.0f);
        return dx * dx + dy * dy;
    };
    int stack[64];
    int ss = 0, cur = 0;
    uint32_t found = kNone, tested = 0;
    while (found == kNone) {
        if (cur < 0) {
            if (ss == 0) break;
            cur = stack[--ss];
        }
        if (visits == 0) {
            found = kGiveUp;
            break;
        }
        --visits;
        const uint32_t c0 = (uint32_t)__ldg(&sep[cur]);
        const uint8_t cl = __ldg(&cil[cur]);
        cur = -1;
        int in[2];
        float dp[2];
        int m = 0;
        for (uint32_t ch = 0; ch < 2; ++ch) {
            const uint32_t c = c0 + ch;
            if (cl & (ch + 1)) {  // leaf: the point itself
                if (c == s.i || c == ga || c == gb || found != kNone) continue;
                if (all && ++tested > kMaxFlatLeaves) {
                    found = kGiveUp;
                    continue;
                }
                const float4 q = __ldg(&s.cm[c]);
                if (hits(q, q) && s.conflict(tr, xy2(q), c)) found = c;
            } else {
                const float4 lo = __ldg(&boxes[c].lo), hi = __ldg(&boxes[c].hi);
                if (hits(lo, hi)) {
                    in[m] = (int)c;
                    dp[m] = dist_p(lo, hi);
                    ++m;
                }
            }
        }
        if (m == 2) {
            const int near = dp[1] < dp[0] ? 1 : 0;
            if (ss < 64) stack[ss++] = in[1 - near];
            else s.st |= ST_STACK_OVERFLOW;
            cur = in[near];
        } else if (m == 1) {
            cur = in[0];
        }
    }
    return found;
}

// Verification sweep.  sweep_all: until every triangle is verified (or the
// star's query budget is spent); otherwise at most one query per triangle
// present at the start.  One star per thread in Morton order (neighbouring
// stars do similar work), and find_intruder leaves its traversal loop at one
// point only: lanes of a warp then stay together far better than with a
// work queue or a return from inside the loop.
__global__ void __launch_bounds__(kM2Block) k_m2_verify(uint32_t n, const float4* __restrict__ cm,
                                                        const int32_t* __restrict__ sep,
                                                        const uint8_t* __restrict__ cil,
                                                        const NodeBox* __restrict__ boxes, uint32_t* loc,
                                                        uint32_t* tri, uint32_t* nloc, uint32_t* ntri,
                                                        uint8_t* done, uint32_t* words, int sweep_all) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (done[i]) continue;
        Star s = load_star(i, n, cm, loc, tri, nloc[i], ntri[i]);
        const uint32_t budget = sweep_all ? kMaxQueries : s.Tl;
        uint32_t queries = 0, ti = 0, visits = kMaxVisits;
        bool stopped = false;
        while (ti < s.Tl) {
            const uint32_t tr = s.T[32 * (size_t)ti];
            if (tr & kVerified) {
                ++ti;
                continue;
            }
            if (queries++ >= budget) {
                stopped = true;
                if (sweep_all) s.st |= ST_WALK_CAP;
                break;
            }
            const uint32_t q = find_intruder(s, tr, sep, cil, boxes, visits);
            if (q == kGiveUp) {
                stopped = true;
                s.st |= ST_WALK_CAP;
                break;
            }
            if (q == kNone) {
                s.T[32 * (size_t)ti] = tr | kVerified;
                ++ti;
                continue;
            }
            if (!s.insert(q) && s.L >= kLocal2) {  // local ids exhausted
                stopped = true;
                break;
            }
            ti = 0;  // triangles moved; verified ones are skipped
        }
        nloc[i] = s.L;
        ntri[i] = s.Tl;
        done[i] = stopped ? 0 : 1;
        if (stopped) atomicAdd(&words[1], 1u);
        if (s.st) atomicOr(&words[0], s.st);
    }
}

// Triangles each point writes: those of its star it is the smallest id of,
// without super nodes when drop_super (mesh.cpp:708-753).
__global__ void k_m2_count(uint32_t n, const uint32_t* __restrict__ loc, const uint32_t* __restrict__ tri,
                           const uint32_t* __restrict__ ntri, int drop_super, uint32_t* __restrict__ nout) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t base = (size_t)(i >> 5) * 32 * kLocal2 + (i & 31);
    uint32_t c = 0;
    const uint32_t Tl = ntri[i];
    for (uint32_t t = 0; t < Tl; ++t) {
        const uint32_t tr = tri[base + 32 * (size_t)t];
        const uint32_t a = tr & 255u, b = (tr >> 8) & 255u;
        if (drop_super && (a < kSuper2 || b < kSuper2)) continue;
        c += (i < loc[base + 32 * (size_t)a] && i < loc[base + 32 * (size_t)b]);
    }
    nout[i] = c;
}

// Compress (mesh.cpp:756-795): (owner, b, c) counter-clockwise, in star order.
__global__ void k_m2_write(uint32_t n, const uint32_t* __restrict__ loc, const uint32_t* __restrict__ tri,
                           const uint32_t* __restrict__ ntri, int drop_super, const uint32_t* __restrict__ elemrow,
                           uint32_t* __restrict__ elems) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t base = (size_t)(i >> 5) * 32 * kLocal2 + (i & 31);
    uint32_t put = elemrow[i];
    const uint32_t Tl = ntri[i];
    for (uint32_t t = 0; t < Tl; ++t) {
        const uint32_t tr = tri[base + 32 * (size_t)t];
        const uint32_t a = tr & 255u, b = (tr >> 8) & 255u;
        if (drop_super && (a < kSuper2 || b < kSuper2)) continue;
        const uint32_t ga = loc[base + 32 * (size_t)a], gb = loc[base + 32 * (size_t)b];
        if (!(i < ga && i < gb)) continue;
        const bool neg = (tr >> 16) & 1u;
        elems[3 * (size_t)put] = i;
        elems[3 * (size_t)put + 1] = neg ? gb : ga;
        elems[3 * (size_t)put + 2] = neg ? ga : gb;
        ++put;
    }
}

}  // namespace

// The lane-interleaved star slots must stay below 2^32 x 4 bytes per array.
constexpr uint32_t kMaxNodesMesh2D = 16u * 1024u * 1024u;

Mesh2D::Mesh2D() {
    SB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    lbvh.fit_point = true;
    lbvh.tail = kSuper2;
    lbvh.bits = 64;
    words.ensure(8);
}

Mesh2D::~Mesh2D() {
    if (stream) cudaStreamDestroy(stream);
}

void Mesh2D::set_nodes_host(uint32_t n, const float* coords) {
    inited = compressed = drop_super = false;
    n_nodes = 0;
    if (n < 2 || n > kMaxNodesMesh2D) throw std::invalid_argument("Mesh2D needs 2 to 16M nodes");
    staging.ensure(2 * (size_t)n);
    SB_CUDA(cudaMemcpyAsync(staging.ptr, coords, sizeof(float) * 2 * (size_t)n, cudaMemcpyHostToDevice, stream));
    input_bad.ensure(1);
    if (any_nonfinite(staging.ptr, 2 * (size_t)n, input_bad.ptr, pinned.h + 12, stream))
        throw std::invalid_argument("Mesh2D::set_nodes: a coordinate is infinite or NaN");
    nodes.ensure(n);
    k_pack_points2d<<<grid_for(n, 256), 256, 0, stream>>>(n, staging.ptr, nodes.ptr);
    SB_LAUNCH_CHECK();
    n_nodes = n;
}

void Mesh2D::init() {
    if (n_nodes < 2) throw std::invalid_argument("Mesh2D::init before set_nodes");
    const uint32_t n = n_nodes;
    SB_CUDA(cudaMemsetAsync(words.ptr, 0, 8 * sizeof(uint32_t), stream));
    lbvh.build(nodes.ptr, n, stream, words.ptr, nullptr);
    k_super2d<<<1, 32, 0, stream>>>(lbvh.bb_glob.ptr, lbvh.obj_m.ptr, n);
    SB_LAUNCH_CHECK();
    const size_t slots = (size_t)((n + 31) / 32) * 32 * kLocal2;
    loc.ensure(slots);
    tri.ensure(slots);
    nloc.ensure(n);
    ntri.ensure(n);
    done.ensure(n);
    k_m2_init<<<grid_for(n, 256), 256, 0, stream>>>(n, lbvh.obj_m.ptr, loc.ptr, tri.ptr, nloc.ptr, ntri.ptr, done.ptr,
                                                    words.ptr);
    SB_LAUNCH_CHECK();
    inited = true;
    compressed = drop_super = false;
}

void Mesh2D::insert_morton_neighbors() {
    if (!inited) throw std::invalid_argument("Mesh2D::insert_morton_neighbors before init");
    k_m2_morton<<<grid_for(n_nodes, kM2Block), kM2Block, 0, stream>>>(n_nodes, lbvh.obj_m.ptr, loc.ptr, tri.ptr,
                                                                      nloc.ptr, ntri.ptr, words.ptr);
    SB_LAUNCH_CHECK();
    compressed = false;
}

static void verify_sweep(Mesh2D& m, int all) {
    if (!m.inited) throw std::invalid_argument("Mesh2D insertion before init");
    const uint32_t n = m.n_nodes;
    SB_CUDA(cudaMemsetAsync(m.words.ptr + 1, 0, sizeof(uint32_t), m.stream));
    k_m2_verify<<<grid_for(n, kM2Block), kM2Block, 0, m.stream>>>(
        n, m.lbvh.obj_m.ptr, m.lbvh.sep.ptr, m.lbvh.cil.ptr, m.lbvh.boxes.ptr, m.loc.ptr, m.tri.ptr, m.nloc.ptr,
        m.ntri.ptr, m.done.ptr, m.words.ptr, all);
    SB_LAUNCH_CHECK();
    m.compressed = false;
}

void Mesh2D::insert_bvh_neighbors() { verify_sweep(*this, 0); }
void Mesh2D::insert_iterative() { verify_sweep(*this, 1); }
void Mesh2D::remove_super_nodes() {
    drop_super = true;
    compressed = false;
}

uint32_t Mesh2D::compress() {
    if (!inited) throw std::invalid_argument("Mesh2D::get_nelem before init");
    const uint32_t n = n_nodes;
    nout.ensure(n);
    elemrow.ensure((size_t)n + 1);
    k_m2_count<<<grid_for(n, 256), 256, 0, stream>>>(n, loc.ptr, tri.ptr, ntri.ptr, drop_super ? 1 : 0, nout.ptr);
    SB_LAUNCH_CHECK();
    exclusive_scan_u32(scan, nout.ptr, elemrow.ptr, n, stream);
    SB_CUDA(cudaMemcpyAsync(pinned.h, elemrow.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    n_elems = pinned.h[0];
    elems.ensure(3 * (size_t)std::max(n_elems, 1u));
    k_m2_write<<<grid_for(n, 256), 256, 0, stream>>>(n, loc.ptr, tri.ptr, ntri.ptr, drop_super ? 1 : 0, elemrow.ptr,
                                                     elems.ptr);
    SB_LAUNCH_CHECK();
    compressed = true;
    return n_elems;
}

void Mesh2D::read_status() {
    SB_CUDA(cudaMemcpyAsync(pinned.h + 8, words.ptr, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    last_status |= pinned.h[8];
    last_incomplete = pinned.h[9];
}

}  // namespace sb
