// 3D direct alpha shape kernels for sm_100a (compiled with -fmad=false so the
// reference's non-exact float tests are evaluated as separate IEEE operations).
#include <algorithm>
#include <cstring>

#include "ashape3d.cuh"
#include "predicates.cuh"

namespace sb {
namespace {

// 2*delta, delta = sqrt((1+5eps)/(1-3eps)) (DirectAlphaShape3D.cpp:196,328).
constexpr float kTwoDelta = 2.0000004768371866248429007339848490744624f;
constexpr int kStarBlock = 64;

struct StarParams {
    uint32_t n;
    const float4* cm;    // Morton-ordered spheres + 4 infinity points
    const uint32_t* cand;
    uint32_t* tets;
    const uint32_t* nineig;
    uint32_t* nout;
    uint32_t* nfneig;
    uint8_t* nkeep;
    uint8_t* node_is_bnd;
    uint4* emask;
    uint4* bmask;
    uint32_t* words;     // status, deferred count, truncated, exact calls
    uint32_t* deferred;  // stars queued for the exact pass: {star, stop state} pairs
};

__device__ __forceinline__ float3 xyz(float4 p) { return make_float3(p.x, p.y, p.z); }

// Infinity points around the global box (DirectAlphaShape3D.cpp:139-171).
__global__ void k_infinity(const float* bb, float4* cm, uint32_t n) {
    if (threadIdx.x != 0) return;
    float avg[3], rg[3];
    for (int k = 0; k < 3; ++k) {
        avg[k] = 0.5f * (bb[3 + k] + bb[k]);
        rg[k] = bb[3 + k] - bb[k];
    }
    const float mr = fmaxf(rg[0], fmaxf(rg[1], rg[2]));
    const float two = 2.0f * mr;
    cm[n + 0] = make_float4(avg[0] - two, avg[1] - two, avg[2] - two, 1.0f);
    cm[n + 1] = make_float4(avg[0] + two, avg[1] - two, avg[2] - two, 1.0f);
    cm[n + 2] = make_float4(avg[0] + two, avg[1] + two, avg[2] - two, 1.0f);
    cm[n + 3] = make_float4(avg[0], avg[1], avg[2] + two, 1.0f);
}

// Candidate neighbours by LBVH depth-first search (fill pass,
// DirectAlphaShape3D.cpp:318-364): child 0 then child 1 are tested at pop
// time, internal children pushed in that order (so child 1 is visited first).
// Stops after the 125th hit: only the first 124 can enter the star.
__global__ void __launch_bounds__(128) k_candidates(const float4* __restrict__ cm, uint32_t n,
                                                    const int32_t* __restrict__ sep, const uint8_t* __restrict__ cil,
                                                    const NodeBox* __restrict__ boxes, uint32_t* __restrict__ cand,
                                                    uint32_t* __restrict__ nineig, uint32_t* words) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= n) return;
    uint32_t* cp = cand + list_base<kCandInterleave, kCandMax>(tid);
    // The reference pushes the intersecting internal children in the order
    // child 0, child 1 and pops the last one next; here that last one is
    // taken directly (no push/pop) and only the other is pushed, so the
    // nodes are visited in the same order with half the stack traffic.
    int stack[64];
    int ss = 0;
    int cur_node = 0;  // root
    bool done = false;
    uint32_t k = 0;
    const float4 si = cm[tid];
    const float rs = kTwoDelta * si.w;
    const float rs2 = rs * rs;
    bool overflow = false;
    while (!done) {
        if (cur_node < 0) {
            if (ss == 0) break;
            cur_node = stack[--ss];
        }
        const uint32_t cur = (uint32_t)cur_node;
        cur_node = -1;
        const uint32_t s = (uint32_t)__ldg(&sep[cur]);
        const uint8_t cl = __ldg(&cil[cur]);
#pragma unroll
        for (uint32_t ch = 0; ch < 2; ++ch) {
            const uint32_t c = s + ch;
            if (!(cl & (ch + 1))) {
                const float4 lo = __ldg(&boxes[c].lo);
                const float4 hi = __ldg(&boxes[c].hi);
                const float dmaxx = fmaxf(si.x - hi.x, 0.0f);
                const float dmaxy = fmaxf(si.y - hi.y, 0.0f);
                const float dmaxz = fmaxf(si.z - hi.z, 0.0f);
                const float dminx = fmaxf(lo.x - si.x, 0.0f);
                const float dminy = fmaxf(lo.y - si.y, 0.0f);
                const float dminz = fmaxf(lo.z - si.z, 0.0f);
                const float d2 = dmaxx * dmaxx + dminx * dminx + dmaxy * dmaxy + dminy * dminy + dmaxz * dmaxz +
                                 dminz * dminz;
                if (d2 < rs2) {
                    if (cur_node >= 0) {  // child 0 goes below child 1 on the stack
                        if (ss < 64) stack[ss++] = cur_node;
                        else overflow = true;
                    }
                    cur_node = (int)c;
                }
            } else if (tid != c) {
                const float4 sj = __ldg(&cm[c]);
                const float ma = fminf(si.w, sj.w);
                const float dx = si.x - sj.x, dy = si.y - sj.y, dz = si.z - sj.z;
                const float d2 = dx * dx + dy * dy + dz * dz;
                const float lim = (kTwoDelta * ma) * (kTwoDelta * ma);
                if (d2 < lim) {
                    if (k < (uint32_t)kCandMax) cp[(size_t)k * kCandInterleave] = c;
                    ++k;
                    if (k > (uint32_t)kCandMax) { done = true; break; }
                }
            }
        }
    }
    nineig[tid] = k + 4 > (uint32_t)kStarCap ? (uint32_t)kStarCap : k + 4;
    if (k > (uint32_t)kCandMax) atomicAdd(&words[2], 1u);
    if (overflow) atomicOr(&words[0], ST_STACK_OVERFLOW);
}

__device__ __forceinline__ uint32_t pack_tet(uint32_t a, uint32_t b, uint32_t c) { return a | (b << 8) | (c << 16); }

// One star: insertion loop (DirectAlphaShape3D.cpp:384-583) and alpha filter
// (:585-693).  With kExact false only predicate stages 1-2 are available: at
// its first undecided test the star stops (returns false) and leaves in
// `state` where it stopped (candidate pi, scan position ti, conflicts R so far,
// tet count Tlast; its tets are in place in P.tets).  With kExact true stage 3
// runs in place, and a non-zero `state` resumes the star there: every test
// before it was decided exactly as stage 3 would have decided it.
// kCount (profiling runs only) also counts the stage-1 tests and stage-2
// evaluations into work[0..1].
template <bool kExact, bool kCount = false>
__device__ bool star_one(const StarParams& P, uint32_t tid, uint8_t* cyc /* stride kStarBlock */, uint32_t& st,
                         uint32_t& nex, uint32_t& state, uint32_t* work = nullptr) {
    const uint32_t n = P.n;
    const uint32_t* cp = P.cand + list_base<kCandInterleave, kCandMax>(tid);
    uint32_t* tp = P.tets + list_base<kTetInterleave, kTetCap>(tid);
#define T(k) tp[(size_t)(k) * kTetInterleave]
#define CYC(j) cyc[(size_t)(j) * kStarBlock]
    auto glob = [&](uint32_t j) -> uint32_t { return j < 4 ? n + j : __ldg(&cp[(size_t)(j - 4) * kCandInterleave]); };
    auto pos = [&](uint32_t g) -> float3 { return xyz(__ldg(&P.cm[g])); };

    if (!state) {
        T(0) = pack_tet(0, 2, 1);
        T(1) = pack_tet(1, 2, 3);
        T(2) = pack_tet(0, 1, 3);
        T(3) = pack_tet(0, 3, 2);
    }
    const uint32_t K = P.nineig[tid];
    if (K - 4 < 3) {
        P.node_is_bnd[tid] = 1;
        P.nout[tid] = 0;
        P.nkeep[tid] = 0;
        P.nfneig[tid] = 0;
        P.emask[tid] = make_uint4(0, 0, 0, 0);
        P.bmask[tid] = make_uint4(0, 0, 0, 0);
        return true;
    }
    const float3 pa = pos(tid);
    uint32_t Tlast = 4, pi0 = 4, ti0 = 0, R0 = 0;
    if (state) {
        pi0 = state & 0xffu;
        ti0 = (state >> 8) & 0xffu;
        R0 = (state >> 16) & 0xffu;
        Tlast = state >> 24;
    }
    for (uint32_t pi = pi0; pi < K; ++pi) {
        const uint32_t q = glob(pi);
        const float3 pe = pos(q);
        uint32_t R = 0, ti = 0;
        if (pi == pi0) {
            R = R0;
            ti = ti0;
        }
        // The next tet word is loaded while the current one is tested: it is
        // T(ti + 1) unless the test finds a conflict, when the swap brings T(Tlast - 1).
        uint32_t t = ti < Tlast ? T(ti) : 0u;
        while (ti < Tlast) {
            const uint32_t tn = ti + 1 < Tlast ? T(ti + 1) : 0u;
            const uint32_t ga = glob(t & 0xffu), gb = glob((t >> 8) & 0xffu), gc = glob((t >> 16) & 0xffu);
            const float3 p[5] = {pa, pos(ga), pos(gb), pos(gc), pe};
            const uint32_t ids[5] = {tid, ga, gb, gc, q};
            float det;
            bool decided;
            if (kCount) {
                ++work[0];
                decided = pred::conflict_fast_count(p, det, work[1]);
            } else {
                decided = pred::conflict_fast(p, det);
            }
            if (!decided) {
                if (!kExact) {  // pi < 128, ti < Tlast <= 252, R <= 252: one byte each
                    state = pi | (ti << 8) | (R << 16) | (Tlast << 24);
                    return false;
                }
                ++nex;
                det = pred::conflict_exact_local(p, ids, st);
            }
            if (det > 0.0f) {
                ++R;
                --Tlast;
                const uint32_t moved = T(Tlast);
                T(ti) = moved;
                T(Tlast) = t;
                t = moved;
            } else {
                ++ti;
                t = tn;
            }
        }
        if (!R) continue;
        for (int j = 0; j < kStarCap; ++j) CYC(j) = 255;
        --R;
        const uint32_t tl = T(Tlast + R);
        const uint32_t la = tl & 0xffu, lb = (tl >> 8) & 0xffu, lc = (tl >> 16) & 0xffu;
        CYC(la) = (uint8_t)lb;
        CYC(lb) = (uint8_t)lc;
        CYC(lc) = (uint8_t)la;
        uint32_t cur = Tlast;
        uint32_t first = la;
        int swap_with = (int)(Tlast + R) - 1;
        int niter = 0;
        // Cavity boundary walk (Ray et al. 2018, Alg. 4 as tailored at :499-574).
        while (R && niter++ < 100) {
            const uint32_t tw = T(cur);
            const uint32_t tc[3] = {tw & 0xffu, (tw >> 8) & 0xffu, (tw >> 16) & 0xffu};
            const uint32_t ty[3] = {CYC(tc[0]), CYC(tc[1]), CYC(tc[2])};
            bool inb[3], opp[3];
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                inb[e] = ty[e] != 255u;
                opp[e] = ty[(e + 1) % 3] == tc[e];
            }
            bool simple = opp[0] || opp[1] || opp[2];
#pragma unroll
            for (int e = 0; e < 3; ++e) simple = simple && (opp[e] || opp[(e + 1) % 3] || !inb[(e + 1) % 3]);
            if (!simple) {
                ++cur;
                if (cur > (uint32_t)swap_with) cur = Tlast;
                continue;
            }
#pragma unroll
            for (int e = 0; e < 3; ++e)
                if (!opp[e]) CYC(tc[e]) = (uint8_t)tc[(e + 1) % 3];
#pragma unroll
            for (int e = 0; e < 3; ++e) {
                if (opp[e] && opp[(e + 1) % 3]) {
                    if (first == tc[(e + 1) % 3]) first = ty[(e + 1) % 3];
                    CYC(tc[(e + 1) % 3]) = 255;
                }
            }
            T(cur) = T(swap_with);
            T(swap_with) = tw;
            --swap_with;
            --R;
            cur = Tlast;
        }
        if (R) st |= ST_WALK_CAP;
        // Fan the new tets around the boundary cycle (:577-582).  A broken
        // cycle (the empty marker 255 reached; undefined behaviour in the
        // reference) stops this star before a tet with the marker is written,
        // so no local id outside the star is ever looked up.
        cur = first;
        int guard = 0;
        bool broken = false;
        do {
            if (cur >= (uint32_t)kStarCap || CYC(cur) >= (uint32_t)kStarCap) {
                st |= ST_BROKEN_CYCLE;
                broken = true;
                break;
            }
            if (Tlast >= (uint32_t)kTetCap || ++guard > kTetCap) {
                st |= ST_TET_CAP;
                broken = true;
                break;
            }
            const uint32_t nx = CYC(cur);
            T(Tlast) = pack_tet(pi, cur, nx);
            ++Tlast;
            cur = nx;
        } while (cur != first);
        if (broken) break;
    }

    // Alpha filter and free-surface flags (:585-693); CYC becomes a counter.
    for (int j = 0; j < kStarCap; ++j) CYC(j) = 0;
    bool bnd = false;
    uint32_t nout = 0, nkeep = 0, ti = 0;
    while (ti < Tlast) {
        const uint32_t t = T(ti);
        const uint32_t la = t & 0xffu, lb = (t >> 8) & 0xffu, lc = (t >> 16) & 0xffu;
        if (la < 4 || lb < 4 || lc < 4) {
            bnd = true;
            --Tlast;
            T(ti) = T(Tlast);
            continue;
        }
        uint32_t i1 = tid, i2 = glob(la), i3 = glob(lb), i4 = glob(lc), x;
        if (i1 > i3) { x = i3; i3 = i1; i1 = x; }
        if (i2 > i4) { x = i4; i4 = i2; i2 = x; }
        if (i1 > i2) { x = i2; i2 = i1; i1 = x; }
        if (i3 > i4) { x = i4; i4 = i3; i3 = x; }
        if (i2 > i3) { x = i3; i3 = i2; i2 = x; }
        const float4 qa = P.cm[i1], qb = P.cm[i2], qc = P.cm[i3], qd = P.cm[i4];
        const float tx = qa.x - qd.x, ty = qa.y - qd.y, tz = qa.z - qd.z;
        const float ux = qb.x - qd.x, uy = qb.y - qd.y, uz = qb.z - qd.z;
        const float vx = qc.x - qd.x, vy = qc.y - qd.y, vz = qc.z - qd.z;
        const float d2t = tx * tx + ty * ty + tz * tz;
        const float d2u = ux * ux + uy * uy + uz * uz;
        const float d2v = vx * vx + vy * vy + vz * vz;
        const float vol = tz * (ux * vy - vx * uy) - uz * (tx * vy - vx * ty) + vz * (tx * uy - ux * ty);
        // |t|^2 u x v + |u|^2 v x t + |v|^2 t x u
        float ax = d2t * (uy * vz - uz * vy), ay = d2t * (uz * vx - ux * vz), az = d2t * (ux * vy - uy * vx);
        ax = ax + d2u * (vy * tz - vz * ty);
        ay = ay + d2u * (vz * tx - vx * tz);
        az = az + d2u * (vx * ty - vy * tx);
        ax = ax + d2v * (ty * uz - tz * uy);
        ay = ay + d2v * (tz * ux - tx * uz);
        az = az + d2v * (tx * uy - ty * ux);
        const float rc = (ax * ax + ay * ay + az * az) / (4.f * vol * vol);
        if (rc <= qa.w * qa.w && rc <= qb.w * qb.w && rc <= qc.w * qc.w && rc <= qd.w * qd.w) {
            CYC(la) = (uint8_t)(CYC(la) + 1);
            CYC(lb) = (uint8_t)(CYC(lb) + 1);
            CYC(lc) = (uint8_t)(CYC(lc) + 1);
            ++nkeep;
            if (tid == i1) {
                ++nout;
                ++ti;
            } else {
                --Tlast;
                T(ti) = T(Tlast);
                T(Tlast) = t;
            }
        } else {
            bnd = true;
            --Tlast;
            T(ti) = T(Tlast);
        }
    }
    uint32_t em[4] = {0, 0, 0, 0}, bm[4] = {0, 0, 0, 0}, nf = 0;
    for (int j = 0; j < kStarCap; ++j) {
        const uint32_t c = CYC(j);
        if (c) {
            em[j >> 5] |= 1u << (j & 31);
            if (c <= 3) bm[j >> 5] |= 1u << (j & 31);
            ++nf;
        }
    }
    P.node_is_bnd[tid] = bnd ? 1 : 0;
    P.nout[tid] = nout;
    P.nkeep[tid] = (uint8_t)nkeep;
    P.nfneig[tid] = nf;
    P.emask[tid] = make_uint4(em[0], em[1], em[2], em[3]);
    P.bmask[tid] = make_uint4(bm[0], bm[1], bm[2], bm[3]);
    return true;
#undef T
#undef CYC
}

// Fast pass, one thread per star, predicate stages 1-2 only; stars that need
// the exact stage are queued for k_star_exact (they are rare and clustered:
// co-spherical lattice sites, near-degenerate blobs).
// Persistent: each lane takes the next star in Morton order from a global
// counter (words[6]) when it finishes one, so a lane whose star is short does
// not idle until the longest star of its warp is done.
__global__ void __launch_bounds__(kStarBlock, 16) k_star(StarParams P) {
    __shared__ uint8_t s_cyc[kStarCap * kStarBlock];
    uint32_t st = 0;
    for (;;) {
        const uint32_t tid = atomicAdd(&P.words[6], 1u);
        if (tid >= P.n) break;
        uint32_t nex = 0, state = 0;
        if (!star_one<false>(P, tid, s_cyc + threadIdx.x, st, nex, state)) {
            const uint32_t g = atomicAdd(&P.words[1], 1u);
            P.deferred[2 * (size_t)g] = tid;
            P.deferred[2 * (size_t)g + 1] = state;
        }
    }
    if (st) atomicOr(&P.words[0], st);
}

// The fast pass with work counters (profiling runs): the same decisions and
// outputs, plus the number of stage-1 tests and stage-2 evaluations summed
// into work64[0..1].
__global__ void __launch_bounds__(kStarBlock, 16) k_star_count(StarParams P, unsigned long long* work64) {
    __shared__ uint8_t s_cyc[kStarCap * kStarBlock];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= P.n) return;
    uint32_t st = 0, nex = 0, state = 0;
    uint32_t work[2] = {0u, 0u};
    if (!star_one<false, true>(P, tid, s_cyc + threadIdx.x, st, nex, state, work)) {
        const uint32_t g = atomicAdd(&P.words[1], 1u);
        P.deferred[2 * (size_t)g] = tid;
        P.deferred[2 * (size_t)g + 1] = state;
    }
    if (st) atomicOr(&P.words[0], st);
    atomicAdd(&work64[0], (unsigned long long)work[0]);
    if (work[1]) atomicAdd(&work64[1], (unsigned long long)work[1]);
}

// Exact pass: thread g resumes queued star g where the fast pass stopped, with
// stage 3 in place (scratch in its own stack frame); threads past the queue
// length exit at once.
__global__ void __launch_bounds__(kStarBlock, 16) k_star_exact(StarParams P) {
    __shared__ uint8_t s_cyc[kStarCap * kStarBlock];
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.words[1]) return;
    uint32_t st = 0, nex = 0, state = P.deferred[2 * (size_t)g + 1];
    star_one<true>(P, P.deferred[2 * (size_t)g], s_cyc + threadIdx.x, st, nex, state);
    if (st) atomicOr(&P.words[0], st);
    if (nex) atomicAdd(&P.words[3], nex);
}

// CSR edges + global tets (compress, DirectAlphaShape3D.cpp:707-743).
__global__ void __launch_bounds__(128) k_compress(uint32_t n, const uint32_t* __restrict__ cand,
                                                  const uint32_t* __restrict__ tets, const uint32_t* __restrict__ nineig,
                                                  const uint4* __restrict__ emask, const uint4* __restrict__ bmask,
                                                  const uint32_t* __restrict__ row, const uint32_t* __restrict__ elemrow,
                                                  uint32_t* __restrict__ neig, uint8_t* __restrict__ edge_is_bnd,
                                                  uint4* __restrict__ elems) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    if (tid >= n) return;
    const uint32_t* cp = cand + list_base<kCandInterleave, kCandMax>(tid);
    const uint32_t* tp = tets + list_base<kTetInterleave, kTetCap>(tid);
    const uint4 e4 = emask[tid], b4 = bmask[tid];
    const uint32_t em[4] = {e4.x, e4.y, e4.z, e4.w}, bm[4] = {b4.x, b4.y, b4.z, b4.w};
    uint32_t put = row[tid];
    const uint32_t K = nineig[tid];
    for (uint32_t j = 4; j < K; ++j) {
        if ((em[j >> 5] >> (j & 31)) & 1u) {
            neig[put] = cp[(size_t)(j - 4) * kCandInterleave];
            edge_is_bnd[put] = (uint8_t)((bm[j >> 5] >> (j & 31)) & 1u);
            ++put;
        }
    }
    const uint32_t e0 = elemrow[tid], e1 = elemrow[tid + 1];
    auto glob = [&](uint32_t j) -> uint32_t { return j < 4 ? n + j : cp[(size_t)(j - 4) * kCandInterleave]; };
    for (uint32_t e = e0, k = 0; e < e1; ++e, ++k) {
        const uint32_t t = tp[(size_t)k * kTetInterleave];
        elems[e] = make_uint4(tid, glob(t & 0xffu), glob((t >> 8) & 0xffu), glob((t >> 16) & 0xffu));
    }
}

__global__ void k_pack_nodes(uint32_t n, const float* __restrict__ coords, const float* __restrict__ alpha,
                             float4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = make_float4(coords[3 * (size_t)i], coords[3 * (size_t)i + 1], coords[3 * (size_t)i + 2], alpha[i]);
}

// Predicate-level check: the full conflict decision (all three stages) for m
// quintuples; pts m x 5 x 3 floats, ids m x 5; one thread each.
__global__ void __launch_bounds__(64) k_conflict_batch(uint32_t m, const float* __restrict__ pts,
                                                       const uint32_t* __restrict__ ids, float* __restrict__ out,
                                                       float* scratch, uint32_t* status) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    float3 p[5];
    uint32_t id[5];
    for (int k = 0; k < 5; ++k) {
        p[k] = make_float3(pts[15 * (size_t)i + 3 * k], pts[15 * (size_t)i + 3 * k + 1], pts[15 * (size_t)i + 3 * k + 2]);
        id[k] = ids[5 * (size_t)i + k];
    }
    uint32_t st = 0, nex = 0;
    bool need;
    out[i] = pred::conflict_det(p, id, scratch + (size_t)i * pred::kInsphereScratchFloats, need, st, nex);
    if (st) atomicOr(status, st);
}

}  // namespace

void conflict_batch_device(uint32_t m, const float* d_pts, const uint32_t* d_ids, float* d_out, uint32_t* d_status,
                           cudaStream_t stream) {
    DeviceBuffer<float> scratch;
    scratch.ensure((size_t)(m ? m : 1) * pred::kInsphereScratchFloats);
    k_conflict_batch<<<grid_for(m, 64), 64, 0, stream>>>(m, d_pts, d_ids, d_out, scratch.ptr, d_status);
    SB_LAUNCH_CHECK();
    SB_CUDA(cudaStreamSynchronize(stream));
}

AlphaShape3D::AlphaShape3D() {
    SB_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    own_stream = true;
    lbvh.fit_point = true;
    lbvh.tail = 4;
    words.ensure(8);
}

AlphaShape3D::~AlphaShape3D() {
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (own_stream && stream) cudaStreamDestroy(stream);
    if (own_stream_saved) cudaStreamDestroy(own_stream_saved);
}

void AlphaShape3D::set_stream(cudaStream_t s) {
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

void AlphaShape3D::mark(int i) {
    if (!profiling) return;
    if (!ev[i]) SB_CUDA(cudaEventCreate(&ev[i]));
    SB_CUDA(cudaEventRecord(ev[i], stream));
}

void AlphaShape3D::collect_profile() {
    if (!profiling) return;
    SB_CUDA(cudaEventSynchronize(ev[S_COUNT]));
    for (int i = 0; i < S_COUNT; ++i) {
        float ms = 0.f;
        SB_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
        stage_ms[i] = ms;
    }
}

void AlphaShape3D::set_nodes_host(uint32_t n, const float* coords, const float* alpha) {
    if (n < 2) throw std::invalid_argument("AlphaShape3D needs at least 2 nodes");
    if (!coords || !alpha) throw std::invalid_argument("AlphaShape3D::set_nodes: null array");
    if (!all_finite(coords, 3 * (size_t)n) || !all_finite(alpha, n)) {
        n_nodes = 0;
        inited = computed = false;
        throw std::invalid_argument("AlphaShape3D::set_nodes: a coordinate or an alpha is infinite or NaN");
    }
    if (!coords || !alpha) throw std::invalid_argument("AlphaShape3D::set_nodes: null array");
    if (!all_finite(coords, 3 * (size_t)n) || !all_finite(alpha, n)) {
        n_nodes = 0;
        inited = computed = false;
        throw std::invalid_argument("AlphaShape3D::set_nodes: a coordinate or an alpha is infinite or NaN");
    }
    DeviceBuffer<float>& tmp = staging;
    tmp.ensure((size_t)4 * n);
    SB_CUDA(cudaMemcpyAsync(tmp.ptr, coords, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, stream));
    SB_CUDA(cudaMemcpyAsync(tmp.ptr + 3 * (size_t)n, alpha, sizeof(float) * n, cudaMemcpyHostToDevice, stream));
    nodes.ensure(n);
    k_pack_nodes<<<grid_for(n, 256), 256, 0, stream>>>(n, tmp.ptr, tmp.ptr + 3 * (size_t)n, nodes.ptr);
    SB_LAUNCH_CHECK();
    n_nodes = n;
    inited = computed = false;
}

void AlphaShape3D::set_nodes_device(uint32_t n, const float4* spheres) {
    if (n < 2) throw std::invalid_argument("AlphaShape3D needs at least 2 nodes");
    nodes.ensure(n);
    SB_CUDA(cudaMemcpyAsync(nodes.ptr, spheres, sizeof(float4) * n, cudaMemcpyDeviceToDevice, stream));
    n_nodes = n;
    inited = computed = false;
}

void AlphaShape3D::init() {
    if (n_nodes < 2) throw std::invalid_argument("AlphaShape3D::init before set_nodes");
    const uint32_t n = n_nodes;
    const size_t W = (n + 31) / 32;
    SB_CUDA(cudaMemsetAsync(words.ptr, 0, 8 * sizeof(uint32_t), stream));
    lbvh.bits = bits;
    mark(S_BBOX_MORTON);
    lbvh.build(nodes.ptr, n, stream, words.ptr, profiling ? this : nullptr);
    k_infinity<<<1, 32, 0, stream>>>(lbvh.bb_glob.ptr, lbvh.obj_m.ptr, n);
    SB_LAUNCH_CHECK();
    cand.ensure(W * kCandMax * 32);
    nineig.ensure(n);
    mark(S_CANDIDATES);
    k_candidates<<<grid_for(n, 128), 128, 0, stream>>>(lbvh.obj_m.ptr, n, lbvh.sep.ptr, lbvh.cil.ptr, lbvh.boxes.ptr,
                                                       cand.ptr, nineig.ptr, words.ptr);
    SB_LAUNCH_CHECK();
    inited = true;
    computed = false;
}

void AlphaShape3D::compute() {
    if (!inited) init();
    const uint32_t n = n_nodes;
    const size_t W = (n + 31) / 32;
    tets.ensure(W * kTetCap * 32);
    nout.ensure(n);
    nfneig.ensure(n);
    nkeep.ensure(n);
    node_is_bnd.ensure(n);
    emask.ensure(n);
    bmask.ensure(n);
    deferred.ensure(2 * (size_t)n);
    elemrow.ensure((size_t)n + 1);
    row.ensure((size_t)n + 1);
    StarParams P{n, lbvh.obj_m.ptr, cand.ptr, tets.ptr, nineig.ptr, nout.ptr, nfneig.ptr, nkeep.ptr,
                 node_is_bnd.ptr, emask.ptr, bmask.ptr, words.ptr, deferred.ptr};
    SB_CUDA(cudaMemsetAsync(words.ptr + 1, 0, sizeof(uint32_t), stream));
    SB_CUDA(cudaMemsetAsync(words.ptr + 6, 0, sizeof(uint32_t), stream));
    mark(S_STAR);
    if (count_work) {
        work.ensure(2);
        SB_CUDA(cudaMemsetAsync(work.ptr, 0, 2 * sizeof(unsigned long long), stream));
        k_star_count<<<grid_for(n, kStarBlock), kStarBlock, 0, stream>>>(P, work.ptr);
    } else {
        const int resident = kNumSMs * 16;  // 16 blocks of 64 per SM at 64 registers
        k_star<<<std::min(grid_for(n, kStarBlock), resident), kStarBlock, 0, stream>>>(P);
    }
    SB_LAUNCH_CHECK();
    mark(S_STAR_EXACT);
    k_star_exact<<<grid_for(n, kStarBlock), kStarBlock, 0, stream>>>(P);
    SB_LAUNCH_CHECK();
    mark(S_SCAN);
    exclusive_scan_u32(scan, nout.ptr, elemrow.ptr, n, stream);
    exclusive_scan_u32(scan, nfneig.ptr, row.ptr, n, stream);
    SB_CUDA(cudaMemcpyAsync(pinned.h, elemrow.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaMemcpyAsync(pinned.h + 1, row.ptr + n, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    n_elems = pinned.h[0];
    n_edges = pinned.h[1];
    elems.ensure(n_elems);
    neig.ensure(n_edges);
    edge_is_bnd.ensure(n_edges);
    mark(S_COMPRESS);
    k_compress<<<grid_for(n, 128), 128, 0, stream>>>(n, cand.ptr, tets.ptr, nineig.ptr, emask.ptr, bmask.ptr, row.ptr,
                                                     elemrow.ptr, neig.ptr, edge_is_bnd.ptr, elems.ptr);
    SB_LAUNCH_CHECK();
    mark(S_COUNT);
    computed = true;
}

void AlphaShape3D::read_counters() {
    SB_CUDA(cudaMemcpyAsync(pinned.h + 8, words.ptr, 4 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
    SB_CUDA(cudaStreamSynchronize(stream));
    last_status = pinned.h[8];
    last_deferred = pinned.h[9];
    last_truncated = pinned.h[10];
    last_exact = pinned.h[11];
}

}  // namespace sb
