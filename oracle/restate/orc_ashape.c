// Oracle (test infrastructure only): plain-C restatement of the reference's
// 3D "direct" alpha shape, src/mesh/DirectAlphaShape3D.cpp:121-743.
//
// Per point (one OpenMP iteration, the reference's one device thread):
//   1. candidate neighbours by an LBVH depth-first search (:318-364), in
//      traversal order, keeping the first 124 (the star holds at most 128
//      local ids including the 4 "infinity" points, :362-363);
//   2. incremental star Delaunay (:380-583): conflict scan with swap-with-last
//      deletion, cavity boundary walk (<= 100 steps), fan re-triangulation;
//   3. alpha filter and free-surface flags (:587-693) with the owner rule;
//   4. scans and compress into CSR edges and global tets (:697-743).
// Outputs use the reference's Morton-ordered point ids.
#include "stream_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CAND_MAX (ORC_STAR_CAP - 4)
#define TET_CAP (2 * CAND_MAX + 4)

// 2*delta, delta = sqrt((1+5eps)/(1-3eps)) (:196, :328).
static const float k_two_delta = 2.0000004768371866248429007339848490744624f;

typedef struct { uint8_t a, b, c; } ltet;

// Neighbour search of one point (count pass :186-232 / fill pass :318-364).
// Returns the number of candidates found (may exceed CAND_MAX; only the first
// CAND_MAX are stored); *stack_err set on traversal-stack overflow.
static uint32_t gather_candidates(uint32_t tid, const float* cm, const int32_t* sep,
                                  const uint8_t* cil, const float* bx, uint32_t* cand,
                                  int* stack_err) {
    int stack[64];
    int ss = 0;
    stack[ss++] = 0;
    uint32_t k = 0;
    const float* si = cm + 4 * (size_t)tid;
    const float rs = k_two_delta * si[3];
    while (ss != 0) {
        const uint32_t cur = (uint32_t)stack[--ss];
        const uint32_t s = (uint32_t)sep[cur];
        const uint8_t cl = cil[cur];
        for (uint32_t ch = 0; ch < 2; ++ch) {
            const uint32_t c = s + ch;
            if (!(cl & (ch + 1))) {
                const float* b = bx + 6 * (size_t)c;
                const float dmaxx = fmaxf(si[0] - b[3], 0.0f);
                const float dmaxy = fmaxf(si[1] - b[4], 0.0f);
                const float dmaxz = fmaxf(si[2] - b[5], 0.0f);
                const float dminx = fmaxf(b[0] - si[0], 0.0f);
                const float dminy = fmaxf(b[1] - si[1], 0.0f);
                const float dminz = fmaxf(b[2] - si[2], 0.0f);
                const float d2 = dmaxx * dmaxx + dminx * dminx + dmaxy * dmaxy + dminy * dminy +
                                 dmaxz * dmaxz + dminz * dminz;
                if (d2 < rs * rs) {
                    if (ss >= 64) { *stack_err = 1; continue; }
                    stack[ss++] = (int)c;
                }
            } else if (tid != c) {
                const float* sj = cm + 4 * (size_t)c;
                const float ma = fminf(si[3], sj[3]);
                const float dx = si[0] - sj[0], dy = si[1] - sj[1], dz = si[2] - sj[2];
                const float d2 = dx * dx + dy * dy + dz * dz;
                const float lim = (k_two_delta * ma) * (k_two_delta * ma);
                if (d2 < lim) {
                    if (k < CAND_MAX) cand[k] = c;
                    ++k;
                    if (k > CAND_MAX) return k;  // the rest cannot enter the star
                }
            }
        }
    }
    return k;
}

static inline uint32_t glob(uint32_t j, uint32_t n, const uint32_t* cand) {
    return j < 4 ? n + j : cand[j - 4];
}

static inline void sub3(const float* a, const float* b, float* o) {
    o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2];
}
static inline float sqn(const float* v) { return v[0] * v[0] + v[1] * v[1] + v[2] * v[2]; }
static inline void cross3(const float* a, const float* b, float* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

typedef struct {
    uint8_t nout, nkeep, bnd;
    uint32_t nfneig, status, n_exact;
} star_result;

// Star Delaunay + alpha filter of one point (:380-693).  T receives the
// owned, kept tets in T[0..nout); act[] the per-local-id edge usage counts.
static star_result star(uint32_t tid, uint32_t n, uint32_t K, const uint32_t* cand,
                        const float* cm, ltet* T, uint8_t* act) {
    star_result r = {0, 0, 0, 0, 0, 0};
    uint8_t cyc[ORC_STAR_CAP];
    memset(act, 0, ORC_STAR_CAP);
    T[0] = (ltet){0, 2, 1};
    T[1] = (ltet){1, 2, 3};
    T[2] = (ltet){0, 1, 3};
    T[3] = (ltet){0, 3, 2};
    if (K - 4 < 3) { r.bnd = 1; return r; }
    uint32_t Tlast = 4;
    for (uint32_t pi = 4; pi < K; ++pi) {
        const uint32_t q = glob(pi, n, cand);
        uint32_t R = 0, ti = 0;
        while (ti < Tlast) {
            const ltet t = T[ti];
            const uint32_t ids[5] = {tid, glob(t.a, n, cand), glob(t.b, n, cand),
                                     glob(t.c, n, cand), q};
            const float* pts[5];
            for (int k = 0; k < 5; ++k) pts[k] = cm + 4 * (size_t)ids[k];
            int ex = 0;
            const float det = orc_conflict_det(pts, ids, &ex);
            r.n_exact += (uint32_t)ex;
            if (det > 0.0f) {
                ++R;
                --Tlast;
                T[ti] = T[Tlast];
                T[Tlast] = t;
            } else {
                ++ti;
            }
        }
        if (!R) continue;
        memset(cyc, 255, sizeof cyc);
        --R;
        const ltet tl = T[Tlast + R];
        cyc[tl.a] = tl.b;
        cyc[tl.b] = tl.c;
        cyc[tl.c] = tl.a;
        uint32_t cur = Tlast;
        uint32_t first = tl.a;
        int swap_with = (int)(Tlast + R) - 1;
        int niter = 0;
        while (R && niter++ < 100) {
            const uint8_t tc[3] = {T[cur].a, T[cur].b, T[cur].c};
            const uint8_t ty[3] = {cyc[tc[0]], cyc[tc[1]], cyc[tc[2]]};
            int inb[3], opp[3];
            for (int e = 0; e < 3; ++e) {
                inb[e] = ty[e] != 255;
                opp[e] = ty[(e + 1) % 3] == tc[e];
            }
            int simple = opp[0] || opp[1] || opp[2];
            for (int e = 0; e < 3; ++e) simple &= (opp[e] || opp[(e + 1) % 3] || !inb[(e + 1) % 3]);
            if (!simple) {
                ++cur;
                if (cur > (uint32_t)swap_with) cur = Tlast;
                continue;
            }
            for (int e = 0; e < 3; ++e)
                if (!opp[e]) cyc[tc[e]] = tc[(e + 1) % 3];
            for (int e = 0; e < 3; ++e) {
                if (opp[e] && opp[(e + 1) % 3]) {
                    if (first == tc[(e + 1) % 3]) first = ty[(e + 1) % 3];
                    cyc[tc[(e + 1) % 3]] = 255;
                }
            }
            T[cur] = T[swap_with];
            T[swap_with] = (ltet){tc[0], tc[1], tc[2]};
            --swap_with;
            --R;
            cur = Tlast;
        }
        if (R) r.status |= ORC_ERR_WALK;
        // The reference's fan (:577-582) writes {pi, cur, cycle[cur]} and then
        // follows cycle[cur]; if the cycle is broken that entry is the empty
        // marker 255 and the reference goes on to read outside its table
        // (undefined behaviour).  Here the star stops before writing a tet
        // with the marker, and the status records it.
        cur = first;
        int guard = 0;
        do {
            if (cur >= ORC_STAR_CAP || cyc[cur] >= ORC_STAR_CAP) { r.status |= ORC_ERR_CYCLE; break; }
            if (Tlast >= TET_CAP || ++guard > TET_CAP) { r.status |= ORC_ERR_CAP; break; }
            const uint8_t nx = cyc[cur];
            T[Tlast++] = (ltet){(uint8_t)pi, (uint8_t)cur, nx};
            cur = nx;
        } while (cur != first);
        if (r.status & (ORC_ERR_CYCLE | ORC_ERR_CAP)) break;
    }

    // Alpha filter (:587-693).
    memset(cyc, 0, sizeof cyc);
    uint32_t ti = 0;
    while (ti < Tlast) {
        const ltet t = T[ti];
        if (t.a < 4 || t.b < 4 || t.c < 4) {
            r.bnd = 1;
            --Tlast;
            T[ti] = T[Tlast];
            continue;
        }
        uint32_t i1 = tid, i2 = glob(t.a, n, cand), i3 = glob(t.b, n, cand), i4 = glob(t.c, n, cand), x;
        if (i1 > i3) { x = i3; i3 = i1; i1 = x; }
        if (i2 > i4) { x = i4; i4 = i2; i2 = x; }
        if (i1 > i2) { x = i2; i2 = i1; i1 = x; }
        if (i3 > i4) { x = i4; i4 = i3; i3 = x; }
        if (i2 > i3) { x = i3; i3 = i2; i2 = x; }
        const float *pa = cm + 4 * (size_t)i1, *pb = cm + 4 * (size_t)i2;
        const float *pc = cm + 4 * (size_t)i3, *pd = cm + 4 * (size_t)i4;
        float tv[3], uv_[3], vv[3];
        sub3(pa, pd, tv);
        sub3(pb, pd, uv_);
        sub3(pc, pd, vv);
        const float d2t = sqn(tv), d2u = sqn(uv_), d2v = sqn(vv);
        const float vol = tv[2] * (uv_[0] * vv[1] - vv[0] * uv_[1]) -
                          uv_[2] * (tv[0] * vv[1] - vv[0] * tv[1]) +
                          vv[2] * (tv[0] * uv_[1] - uv_[0] * tv[1]);
        float c1[3], c2[3], c3[3], acc[3];
        cross3(uv_, vv, c1);
        cross3(vv, tv, c2);
        cross3(tv, uv_, c3);
        for (int k = 0; k < 3; ++k) acc[k] = d2t * c1[k];
        for (int k = 0; k < 3; ++k) acc[k] = acc[k] + d2u * c2[k];
        for (int k = 0; k < 3; ++k) acc[k] = acc[k] + d2v * c3[k];
        const float rc = sqn(acc) / (4.f * vol * vol);
        if (rc <= pa[3] * pa[3] && rc <= pb[3] * pb[3] && rc <= pc[3] * pc[3] && rc <= pd[3] * pd[3]) {
            act[t.a] += 1;
            act[t.b] += 1;
            act[t.c] += 1;
            cyc[t.a]++;
            cyc[t.b]++;
            cyc[t.c]++;
            r.nkeep++;
            if (tid == i1) {
                r.nout++;
                ++ti;
            } else {
                --Tlast;
                T[ti] = T[Tlast];
                T[Tlast] = t;
            }
        } else {
            r.bnd = 1;
            --Tlast;
            T[ti] = T[Tlast];
        }
    }
    for (int i = 0; i < ORC_STAR_CAP; ++i) r.nfneig += (cyc[i] != 0);
    return r;
}

int orc_ashape3d(uint32_t n, const float* coords, const float* alpha, int bits, orc_ashape* out) {
    memset(out, 0, sizeof *out);
    if (n < 2) return 1;
    out->n = n;
    float* s = (float*)malloc((size_t)n * 16);
    for (uint32_t i = 0; i < n; ++i) {
        s[4 * i] = coords[3 * i];
        s[4 * i + 1] = coords[3 * i + 1];
        s[4 * i + 2] = coords[3 * i + 2];
        s[4 * i + 3] = alpha[i];
    }
    float bb[6];
    int32_t* sep = (int32_t*)malloc((size_t)n * 4);
    uint8_t* cil = (uint8_t*)malloc(n);
    float* bx = (float*)malloc((size_t)n * 24);
    out->perm = (uint32_t*)malloc((size_t)n * 4);
    out->coords_m = (float*)malloc((size_t)(n + 4) * 16);
    orc_lbvh3d(n, s, bits, 1, bb, NULL, out->perm, sep, cil, NULL, NULL, bx, out->coords_m);
    free(s);

    // Infinity points from the global box (:139-171).
    float* cm = out->coords_m;
    {
        float avg[3], rg[3];
        for (int k = 0; k < 3; ++k) { avg[k] = 0.5f * (bb[3 + k] + bb[k]); rg[k] = bb[3 + k] - bb[k]; }
        const float mr = fmaxf(rg[0], fmaxf(rg[1], rg[2]));
        const float two = 2 * mr;
        const float inf[4][3] = {{avg[0] - two, avg[1] - two, avg[2] - two},
                                 {avg[0] + two, avg[1] - two, avg[2] - two},
                                 {avg[0] + two, avg[1] + two, avg[2] - two},
                                 {avg[0], avg[1], avg[2] + two}};
        for (int j = 0; j < 4; ++j) {
            float* p = cm + 4 * (size_t)(n + j);
            p[0] = inf[j][0]; p[1] = inf[j][1]; p[2] = inf[j][2]; p[3] = 1.0f;
        }
    }

    out->nineig = (uint32_t*)malloc((size_t)n * 4);
    out->cand = (uint32_t*)malloc((size_t)n * CAND_MAX * 4);
    out->node_is_bnd = (uint8_t*)malloc(n);
    out->nelem = (uint8_t*)malloc(n);
    ltet* T = (ltet*)malloc((size_t)n * TET_CAP * sizeof(ltet));
    uint8_t* act = (uint8_t*)malloc((size_t)n * ORC_STAR_CAP);
    uint8_t* nout = (uint8_t*)malloc(n);
    uint32_t* nf = (uint32_t*)malloc((size_t)n * 4);
    uint32_t status = 0, ntrunc = 0, nexact = 0;

#pragma omp parallel for schedule(dynamic, 64) reduction(| : status) reduction(+ : ntrunc, nexact)
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t* cd = out->cand + (size_t)i * CAND_MAX;
        for (int j = 0; j < CAND_MAX; ++j) cd[j] = 0xFFFFFFFFu;
        int serr = 0;
        const uint32_t k = gather_candidates(i, cm, sep, cil, bx, cd, &serr);
        if (serr) status |= ORC_ERR_STACK;
        if (k > CAND_MAX) ntrunc++;
        const uint32_t K = (k + 4 > ORC_STAR_CAP) ? ORC_STAR_CAP : k + 4;
        out->nineig[i] = K;
        star_result sr = star(i, n, K, cd, cm, T + (size_t)i * TET_CAP, act + (size_t)i * ORC_STAR_CAP);
        status |= sr.status;
        nexact += sr.n_exact;
        out->node_is_bnd[i] = sr.bnd;
        out->nelem[i] = sr.nkeep;
        nout[i] = sr.nout;
        nf[i] = sr.nfneig;
    }

    out->elemrow = (uint32_t*)malloc((size_t)(n + 1) * 4);
    out->row = (uint32_t*)malloc((size_t)(n + 1) * 4);
    out->elemrow[0] = 0;
    out->row[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        out->elemrow[i + 1] = out->elemrow[i] + nout[i];
        out->row[i + 1] = out->row[i] + nf[i];
    }
    out->n_elems = out->elemrow[n];
    out->n_edges = out->row[n];
    out->elems = (uint32_t*)malloc((size_t)out->n_elems * 16 + 16);
    out->neig = (uint32_t*)malloc((size_t)out->n_edges * 4 + 4);
    out->edge_is_bnd = (uint8_t*)malloc((size_t)out->n_edges + 1);

    // compress (:707-743)
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t* cd = out->cand + (size_t)i * CAND_MAX;
        const uint8_t* a = act + (size_t)i * ORC_STAR_CAP;
        uint32_t put = out->row[i];
        for (uint32_t j = 4; j < out->nineig[i]; ++j) {
            if (a[j]) {
                out->edge_is_bnd[put] = (a[j] <= 3);
                out->neig[put++] = cd[j - 4];
            }
        }
        const ltet* t = T + (size_t)i * TET_CAP;
        for (uint32_t e = out->elemrow[i], k = 0; e < out->elemrow[i + 1]; ++e, ++k) {
            uint32_t* o = out->elems + 4 * (size_t)e;
            o[0] = i;
            o[1] = glob(t[k].a, n, cd);
            o[2] = glob(t[k].b, n, cd);
            o[3] = glob(t[k].c, n, cd);
        }
    }
    out->status = status;
    out->n_truncated = ntrunc;
    out->n_exact = nexact;
    free(sep); free(cil); free(bx); free(T); free(act); free(nout); free(nf);
    return 0;
}

void orc_ashape3d_free(orc_ashape* a) {
    free(a->perm); free(a->coords_m); free(a->nineig); free(a->cand); free(a->elemrow);
    free(a->elems); free(a->row); free(a->neig); free(a->edge_is_bnd); free(a->node_is_bnd);
    free(a->nelem);
    memset(a, 0, sizeof *a);
}

void orc_conflict_batch(uint32_t m, const float* pts, const uint32_t* ids, float* out,
                        uint8_t* used_exact) {
#pragma omp parallel for schedule(static)
    for (uint32_t i = 0; i < m; ++i) {
        const float* p[5];
        for (int k = 0; k < 5; ++k) p[k] = pts + 15 * (size_t)i + 3 * k;
        int ex = 0;
        out[i] = orc_conflict_det(p, ids + 5 * (size_t)i, &ex);
        if (used_exact) used_exact[i] = (uint8_t)ex;
    }
}
