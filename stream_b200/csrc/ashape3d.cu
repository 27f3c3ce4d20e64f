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
    uint32_t* words;     // status, deferred count, truncated, exact calls; [4] exact-pass queue, [6] fast-pass queue
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
// True when a packed tet has an infinity vertex (local id < 4, the upper six
// bits of its byte zero): a zero-byte test on those bits of the three bytes.
__device__ __forceinline__ bool has_infinity(uint32_t t) {
    const uint32_t v = (t >> 2) & 0x3f3f3fu;
    return ((v - 0x010101u) & ~v & 0x808080u) != 0u;
}

// One star: insertion loop (DirectAlphaShape3D.cpp:384-583) and alpha filter
// (:585-693).  With kExact false only predicate stages 1-2 are available: at
// its first undecided test the star stops (returns false) and leaves in
// `state` where it stopped (candidate pi, scan position ti, conflicts R so far,
// tet count Tlast; its tets are in place in P.tets).  With kExact true stage 3
// runs in place, and a non-zero `state` resumes the star there: every test
// before it was decided exactly as stage 3 would have decided it.
// A test whose tet has only finite vertices first compares the filter's
// determinant with a per-star bound of its error bound (star_filter_bound):
// above it the filter is certain without its permanent; otherwise the full
// stages 1-2 run.  The decisions are those of stages 1-2 either way.
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
    // Largest coordinate offset of a finite local point from the centre: the
    // bound under which a test with finite vertices skips the permanent.
    float mc = 0.0f;
    for (uint32_t j = 4; j < K; ++j) {
        const float3 q = pos(glob(j));
        mc = fmaxf(mc, fmaxf(fabsf(q.x - pa.x), fmaxf(fabsf(q.y - pa.y), fabsf(q.z - pa.z))));
    }
    const float fbound = pred::star_filter_bound(mc);
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
            if (kCount) ++work[0];
            float det = -pred::insphere32_det(p[0], p[1], p[2], p[3], p[4]);
            bool decided = fabsf(det) > fbound && !has_infinity(t);
            if (!decided) {
                if (kCount) decided = pred::conflict_fast_count(p, det, work[1]);
                else decided = pred::conflict_fast(p, det);
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
// the exact stage are queued for k_star_exact_coop (they are rare and clustered:
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

// ---------------------------------------------------------------------------
// Exact pass, 8 lanes per queued star (4 stars per warp, in lockstep): the
// star's local points and tets sit in shared memory; each insertion's
// conflict tests are split over the 8 lanes (a test does not depend on where
// its tet sits; undecided ones take stage 3 in the lane), then the group
// leader replays the reference's swap-with-last scan (:484-494) on the
// conflict flags and runs the cavity walk and the fan as star_one does.  The
// first insertion resumes where the fast pass stopped: its scan continues at
// position ti with the R conflicts already found.  The alpha filter is split
// the same way, with the owner-first compaction replayed on the flags.
constexpr int kCoopBlock = 128;  // 4 warps, 16 stars
constexpr uint32_t kFull = 0xffffffffu;

struct CoopStar {
    uint32_t T[kTetCap];         // local tets (3 local ids packed)
    float4 pts[kStarCap];        // x, y, z, alpha of local ids (0..3: infinity points)
    uint32_t flags[8];           // one bit per tet slot
    uint32_t cyc[kStarCap / 4];  // cavity cycle (bytes), then kept-tet counters (bytes)
};
static_assert(sizeof(CoopStar) % 16 == 0, "star records stay 16-byte aligned");

// The reference's scan over slots [ti, N) with conflict flags fw (by original
// slot) and R conflicts already moved past N: a flagged slot is swapped with
// the last live slot, whose tet is tested next at the same position.
// Returns the live count; R grows by the flagged count.
__device__ __forceinline__ uint32_t replay_scan(uint32_t* T, const uint32_t* fw, uint32_t ti, uint32_t N,
                                                uint32_t& R) {
    uint32_t last = N;
    for (;;) {
        uint32_t c = last;  // first flagged original slot in [ti, last)
        for (uint32_t w = ti >> 5; 32u * w < last; ++w) {
            uint32_t m = fw[w];
            if (ti > 32u * w) m &= ~0u << (ti - 32u * w);
            if (m) {
                c = 32u * w + (uint32_t)__ffs(m) - 1u;
                break;
            }
        }
        if (c >= last) break;
        ti = c;
        uint32_t x = T[ti];
        for (;;) {
            --last;
            ++R;
            if (last == ti) {
                T[ti] = x;
                break;
            }
            const uint32_t y = T[last], yf = (fw[last >> 5] >> (last & 31u)) & 1u;
            T[last] = x;
            if (yf) {
                x = y;
                continue;
            }
            T[ti] = y;
            ++ti;
            break;
        }
    }
    return last;
}

__device__ __forceinline__ uint32_t cyc_get(const uint32_t* cyc, uint32_t j) {
    return (cyc[j >> 2] >> (8u * (j & 3u))) & 0xffu;
}
__device__ __forceinline__ void cyc_set(uint32_t* cyc, uint32_t j, uint32_t v) {
    const uint32_t s = 8u * (j & 3u);
    cyc[j >> 2] = (cyc[j >> 2] & ~(0xffu << s)) | (v << s);
}

__global__ void __launch_bounds__(kCoopBlock) k_star_exact_coop(StarParams P) {
    extern __shared__ __align__(16) unsigned char coop_smem[];
    const uint32_t lane = threadIdx.x & 31u, g = lane >> 3, j = lane & 7u;
    CoopStar& S = reinterpret_cast<CoopStar*>(coop_smem)[(threadIdx.x >> 5) * 4 + g];
    const uint32_t n = P.n, nd = P.words[1];
    const uint32_t leader = g * 8u;
    uint32_t st = 0, nex = 0;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&P.words[4], 4u);
        base = __shfl_sync(kFull, base, 0);
        if (base >= nd) break;
        const bool live = base + g < nd;
        const uint32_t tid = live ? P.deferred[2 * (size_t)(base + g)] : 0u;
        const uint32_t state = live ? P.deferred[2 * (size_t)(base + g) + 1] : 0u;
        const uint32_t* cp = P.cand + list_base<kCandInterleave, kCandMax>(tid);
        uint32_t* tp = P.tets + list_base<kTetInterleave, kTetCap>(tid);
        auto glob = [&](uint32_t l) -> uint32_t {
            return l < 4 ? n + l : __ldg(&cp[(size_t)(l - 4) * kCandInterleave]);
        };
        const uint32_t K = live ? P.nineig[tid] : 4u;
        uint32_t pi0 = state & 0xffu, ti0 = (state >> 8) & 0xffu, R0 = (state >> 16) & 0xffu;
        uint32_t Tlast = state >> 24;
        bool work = live;
        float4 pa4 = make_float4(0.f, 0.f, 0.f, 0.f);
        if (work) {
            pa4 = __ldg(&P.cm[tid]);
            for (uint32_t l = j; l < K; l += 8) S.pts[l] = __ldg(&P.cm[glob(l)]);
            for (uint32_t k = j; k < Tlast + R0; k += 8) S.T[k] = tp[(size_t)k * kTetInterleave];
        }
        __syncwarp();
        const float3 pa = xyz(pa4);
        for (uint32_t pi = live ? pi0 : 0;; ++pi) {
            const bool act = work && pi < K;
            if (!__any_sync(kFull, act)) break;
            const bool first_ins = act && pi == pi0;
            const uint32_t t0 = first_ins ? ti0 : 0u;
            uint32_t R = first_ins ? R0 : 0u;
            // ---- conflict tests of slots [t0, Tlast), 8 at a time per star
            const float3 pe = act ? xyz(S.pts[pi]) : pa;
            const uint32_t qg = act ? glob(pi) : 0u;
            const uint32_t r0 = t0 >> 3;
            const uint32_t rounds = act ? (Tlast + 7u) >> 3 : 0u;
            const uint32_t maxr = __reduce_max_sync(kFull, rounds);
            if (j == 0 && act)
                for (int w = 0; w < 8; ++w) S.flags[w] = 0u;
            __syncwarp();
            for (uint32_t r = __reduce_min_sync(kFull, act ? r0 : 0xffffffu); r < maxr; ++r) {
                const uint32_t k = 8u * r + j;
                bool conf = false;
                if (act && k >= t0 && k < Tlast) {
                    const uint32_t t = S.T[k];
                    const uint32_t la = t & 0xffu, lb = (t >> 8) & 0xffu, lc = (t >> 16) & 0xffu;
                    const float3 p[5] = {pa, xyz(S.pts[la]), xyz(S.pts[lb]), xyz(S.pts[lc]), pe};
                    float det;
                    if (!pred::conflict_fast(p, det)) {
                        const uint32_t ids[5] = {tid, glob(la), glob(lb), glob(lc), qg};
                        ++nex;
                        det = pred::conflict_exact_local(p, ids, st);
                    }
                    conf = det > 0.0f;
                }
                const uint32_t cb = __ballot_sync(kFull, conf);
                if (j == 0 && act) reinterpret_cast<uint8_t*>(S.flags)[r] = (uint8_t)(cb >> leader);
            }
            __syncwarp();
            // ---- the leader replays the scan, walks the cavity and fans
            if (j == 0 && act) {
                Tlast = replay_scan(S.T, S.flags, t0, Tlast, R);
                if (R) {
                    uint32_t* cyc = S.cyc;
                    for (int w = 0; w < kStarCap / 4; ++w) cyc[w] = 0xffffffffu;
                    --R;
                    const uint32_t tl = S.T[Tlast + R];
                    const uint32_t la = tl & 0xffu, lb = (tl >> 8) & 0xffu, lc = (tl >> 16) & 0xffu;
                    cyc_set(cyc, la, lb);
                    cyc_set(cyc, lb, lc);
                    cyc_set(cyc, lc, la);
                    uint32_t cur = Tlast;
                    uint32_t first = la;
                    int swap_with = (int)(Tlast + R) - 1;
                    int niter = 0;
                    while (R && niter++ < 100) {
                        const uint32_t tw = S.T[cur];
                        const uint32_t tc[3] = {tw & 0xffu, (tw >> 8) & 0xffu, (tw >> 16) & 0xffu};
                        const uint32_t ty[3] = {cyc_get(cyc, tc[0]), cyc_get(cyc, tc[1]), cyc_get(cyc, tc[2])};
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
                            if (!opp[e]) cyc_set(cyc, tc[e], tc[(e + 1) % 3]);
#pragma unroll
                        for (int e = 0; e < 3; ++e) {
                            if (opp[e] && opp[(e + 1) % 3]) {
                                if (first == tc[(e + 1) % 3]) first = ty[(e + 1) % 3];
                                cyc_set(cyc, tc[(e + 1) % 3], 255u);
                            }
                        }
                        S.T[cur] = S.T[swap_with];
                        S.T[swap_with] = tw;
                        --swap_with;
                        --R;
                        cur = Tlast;
                    }
                    if (R) st |= ST_WALK_CAP;
                    cur = first;
                    int guard = 0;
                    do {
                        if (cur >= (uint32_t)kStarCap || cyc_get(cyc, cur) >= (uint32_t)kStarCap) {
                            st |= ST_BROKEN_CYCLE;
                            work = false;  // this star stops inserting (as star_one)
                            break;
                        }
                        if (Tlast >= (uint32_t)kTetCap || ++guard > kTetCap) {
                            st |= ST_TET_CAP;
                            work = false;
                            break;
                        }
                        const uint32_t nx = cyc_get(cyc, cur);
                        S.T[Tlast] = pack_tet(pi, cur, nx);
                        ++Tlast;
                        cur = nx;
                    } while (cur != first);
                }
            }
            Tlast = __shfl_sync(kFull, Tlast, leader);
            work = __shfl_sync(kFull, work, leader);
            __syncwarp();
        }
        // ---- alpha filter and free-surface flags (:585-693)
        const bool filt = live;
        for (uint32_t w = j; w < kStarCap / 4; w += 8) S.cyc[w] = 0u;
        __syncwarp();
        const uint32_t rounds = filt ? (Tlast + 7u) >> 3 : 0u;
        const uint32_t maxr = __reduce_max_sync(kFull, rounds);
        uint32_t nkeep = 0, nout = 0;
        bool bnd = false;
        for (uint32_t r = 0; r < maxr; ++r) {
            const uint32_t k = 8u * r + j;
            bool keep = false, owner = false, drop = false;
            if (filt && k < Tlast) {
                const uint32_t t = S.T[k];
                const uint32_t la = t & 0xffu, lb = (t >> 8) & 0xffu, lc = (t >> 16) & 0xffu;
                if (la < 4 || lb < 4 || lc < 4) {
                    drop = true;
                } else {
                    // the 4 vertices ordered by global id (the reference's sort)
                    uint32_t i1 = tid, i2 = glob(la), i3 = glob(lb), i4 = glob(lc), x;
                    uint32_t l1 = 255u, l2 = la, l3 = lb, l4 = lc, y;
                    if (i1 > i3) { x = i3; i3 = i1; i1 = x; y = l3; l3 = l1; l1 = y; }
                    if (i2 > i4) { x = i4; i4 = i2; i2 = x; y = l4; l4 = l2; l2 = y; }
                    if (i1 > i2) { x = i2; i2 = i1; i1 = x; y = l2; l2 = l1; l1 = y; }
                    if (i3 > i4) { x = i4; i4 = i3; i3 = x; y = l4; l4 = l3; l3 = y; }
                    if (i2 > i3) { x = i3; i3 = i2; i2 = x; y = l3; l3 = l2; l2 = y; }
                    auto pt = [&](uint32_t l) -> float4 { return l == 255u ? pa4 : S.pts[l]; };
                    const float4 qa = pt(l1), qb = pt(l2), qc = pt(l3), qd = pt(l4);
                    const float tx = qa.x - qd.x, ty = qa.y - qd.y, tz = qa.z - qd.z;
                    const float ux = qb.x - qd.x, uy = qb.y - qd.y, uz = qb.z - qd.z;
                    const float vx = qc.x - qd.x, vy = qc.y - qd.y, vz = qc.z - qd.z;
                    const float d2t = tx * tx + ty * ty + tz * tz;
                    const float d2u = ux * ux + uy * uy + uz * uz;
                    const float d2v = vx * vx + vy * vy + vz * vz;
                    const float vol = tz * (ux * vy - vx * uy) - uz * (tx * vy - vx * ty) + vz * (tx * uy - ux * ty);
                    float ax = d2t * (uy * vz - uz * vy), ay = d2t * (uz * vx - ux * vz), az = d2t * (ux * vy - uy * vx);
                    ax = ax + d2u * (vy * tz - vz * ty);
                    ay = ay + d2u * (vz * tx - vx * tz);
                    az = az + d2u * (vx * ty - vy * tx);
                    ax = ax + d2v * (ty * uz - tz * uy);
                    ay = ay + d2v * (tz * ux - tx * uz);
                    az = az + d2v * (tx * uy - ty * ux);
                    const float rc = (ax * ax + ay * ay + az * az) / (4.f * vol * vol);
                    if (rc <= qa.w * qa.w && rc <= qb.w * qb.w && rc <= qc.w * qc.w && rc <= qd.w * qd.w) {
                        keep = true;
                        owner = tid == i1;
                        atomicAdd(&S.cyc[la >> 2], 1u << (8u * (la & 3u)));
                        atomicAdd(&S.cyc[lb >> 2], 1u << (8u * (lb & 3u)));
                        atomicAdd(&S.cyc[lc >> 2], 1u << (8u * (lc & 3u)));
                    } else {
                        drop = true;
                    }
                }
            }
            const uint32_t kb = __ballot_sync(kFull, keep), ob = __ballot_sync(kFull, keep && owner);
            const uint32_t db = __ballot_sync(kFull, drop);
            nkeep += __popc((kb >> leader) & 0xffu);
            nout += __popc((ob >> leader) & 0xffu);
            bnd = bnd || ((db >> leader) & 0xffu);
            // moved: every slot that is not an owner-kept tet
            if (j == 0 && filt) reinterpret_cast<uint8_t*>(S.flags)[r] = (uint8_t)~(ob >> leader);
        }
        __syncwarp();
        if (j == 0 && filt) {
            uint32_t R = 0;
            const uint32_t front = replay_scan(S.T, S.flags, 0u, Tlast, R);
            if (front != nout) st |= ST_TET_CAP;  // cannot happen: the owner-kept count is the live count
        }
        __syncwarp();
        if (filt) {
            // masks of used local ids (edges) and of ids used by at most 3 kept tets
            uint32_t em[4] = {0, 0, 0, 0}, bm[4] = {0, 0, 0, 0};
#pragma unroll
            for (uint32_t m = 0; m < kStarCap / 8; ++m) {
                const uint32_t l = 8u * m + j, c = cyc_get(S.cyc, l);
                if (c) {
                    em[l >> 5] |= 1u << (l & 31u);
                    if (c <= 3u) bm[l >> 5] |= 1u << (l & 31u);
                }
            }
#pragma unroll
            for (int w = 0; w < 4; ++w)
#pragma unroll
                for (int o = 4; o > 0; o >>= 1) {
                    em[w] |= __shfl_xor_sync(0xffu << leader, em[w], o, 8);
                    bm[w] |= __shfl_xor_sync(0xffu << leader, bm[w], o, 8);
                }
            for (uint32_t k = j; k < nout; k += 8) tp[(size_t)k * kTetInterleave] = S.T[k];
            if (j == 0) {
                P.node_is_bnd[tid] = bnd ? 1 : 0;
                P.nout[tid] = nout;
                P.nkeep[tid] = (uint8_t)nkeep;
                P.nfneig[tid] = __popc(em[0]) + __popc(em[1]) + __popc(em[2]) + __popc(em[3]);
                P.emask[tid] = make_uint4(em[0], em[1], em[2], em[3]);
                P.bmask[tid] = make_uint4(bm[0], bm[1], bm[2], bm[3]);
            }
        }
        __syncwarp();
    }
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
    // The finiteness check runs on the staged copy, and a non-finite input is
    // refused before any meshing kernel runs.
    DeviceBuffer<float>& tmp = staging;
    tmp.ensure((size_t)4 * n);
    SB_CUDA(cudaMemcpyAsync(tmp.ptr, coords, sizeof(float) * 3 * (size_t)n, cudaMemcpyHostToDevice, stream));
    SB_CUDA(cudaMemcpyAsync(tmp.ptr + 3 * (size_t)n, alpha, sizeof(float) * n, cudaMemcpyHostToDevice, stream));
    input_bad.ensure(1);
    if (any_nonfinite(tmp.ptr, (size_t)4 * n, input_bad.ptr, pinned.h + 12, stream)) {
        n_nodes = 0;
        inited = computed = false;
        throw std::invalid_argument("AlphaShape3D::set_nodes: a coordinate or an alpha is infinite or NaN");
    }
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
    SB_CUDA(cudaMemsetAsync(words.ptr + 4, 0, sizeof(uint32_t), stream));
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
    {
        const int smem = 16 * (int)sizeof(CoopStar);
        static std::atomic<uint64_t> coop_attr{0};  // one bit per device
        if (once_per_device(coop_attr))
            SB_CUDA(cudaFuncSetAttribute(k_star_exact_coop, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        int per_sm = 0;
        SB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_star_exact_coop, kCoopBlock, smem));
        k_star_exact_coop<<<std::max(1, per_sm) * kNumSMs, kCoopBlock, smem, stream>>>(P);
        SB_LAUNCH_CHECK();
    }
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
