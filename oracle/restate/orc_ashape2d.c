// Oracle (test infrastructure only): plain-C restatement of the reference's
// 2D "direct" alpha shape, src/mesh/DirectAlphaShape2D.cpp:121-690.
//
// Per point (one OpenMP iteration, the reference's one device thread):
//   1. neighbours by an LBVH depth-first search (:178-224 count, :310-357
//      fill) in traversal order; the fill stops once more than 250 local ids
//      are held (:351-354);
//   2. incremental star Delaunay (:373-515): conflict scan with swap-with-last
//      deletion, the cavity's vertices as a parity bitset, new triangles
//      (r, ni) for its set bits in increasing order;
//   3. infinity removal, alpha filter (circumradius against the smallest
//      alpha) and boundary flags (:528-595) with the owner rule;
//   4. scans and compress into CSR edges and global triangles (:602-690).
// Outputs use the reference's Morton-ordered point ids.
#include "stream_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define N_INF 3
#define FILL_LIMIT 250
// 2*delta, delta = sqrt((1+4eps)/(1-3eps)) (:185-188, :318-320).
static const float k_two_delta2 = 2.0000004172325445139859201780136934301654f;

static inline int box_hit(const float* c, float rs, const float* b) {
    // b: min x, min y, (z), max x, max y, (z) as the 3D box layout of orc_fit
    const float dmaxx = fmaxf(c[0] - b[3], 0.0f);
    const float dmaxy = fmaxf(c[1] - b[4], 0.0f);
    const float dminx = fmaxf(b[0] - c[0], 0.0f);
    const float dminy = fmaxf(b[1] - c[1], 0.0f);
    return dmaxx * dmaxx + dminx * dminx + dmaxy * dmaxy + dminy * dminy < rs * rs;
}

static inline float sqn2(float x, float y) {
    float s = 0.0f;
    s += x * x;
    s += y * y;
    return s;
}

// Neighbour search of point tid.  fill = 0: count all (:178-224); fill = 1:
// store up to the fill limit (:310-357).  Returns the number of neighbours
// (fill: including the 3 infinity ids).
static uint32_t neighbours(uint32_t tid, const float* cm, const int32_t* sep, const uint8_t* cil,
                           const float* boxes, int fill, uint32_t* out, uint32_t* err) {
    int stack[64];
    int ss = 0;
    stack[ss++] = 0;
    const float* si = cm + 4 * (size_t)tid;
    const float rs = k_two_delta2 * si[3];
    uint32_t cnt = fill ? N_INF : 0;
    while (ss != 0) {
        const uint32_t cur = (uint32_t)stack[--ss];
        const uint32_t s = (uint32_t)sep[cur];
        const uint8_t cl = cil[cur];
        for (uint32_t ch = 0; ch < 2; ++ch) {
            if (!(cl & (ch + 1))) {
                if (box_hit(si, rs, boxes + 6 * (size_t)(s + ch))) {
                    if (ss >= 64) { *err |= ORC_ERR_STACK; return cnt; }
                    stack[ss++] = (int)(s + ch);
                }
            } else if (s + ch != tid || !fill) {
                const float* sj = cm + 4 * (size_t)(s + ch);
                const float ma = fminf(si[3], sj[3]);
                const int hit = sqn2(si[0] - sj[0], si[1] - sj[1]) < (k_two_delta2 * ma) * (k_two_delta2 * ma);
                if (!fill) {
                    cnt += hit && (tid != s + ch);
                } else if (hit) {
                    out[cnt - N_INF] = s + ch;
                    cnt++;
                }
            }
        }
        if (fill && cnt > FILL_LIMIT) break;
    }
    return cnt;
}

typedef struct { uint8_t a, b; } tri2;

static inline uint32_t gid(uint32_t j, uint32_t n, const uint32_t* nb) { return j < N_INF ? n + j : nb[j - N_INF]; }

// In-circle decision of the reference's star kernel (:437-479), sign only:
// > 0 when the inserted point conflicts with the local triangle (si, b, c).
static float conflict2(const float* cm, uint32_t i1, uint32_t i2, uint32_t i3, uint32_t i4, uint32_t* n_exact) {
    const float *pa = cm + 4 * (size_t)i1, *pb = cm + 4 * (size_t)i2, *pc = cm + 4 * (size_t)i3,
                *pd = cm + 4 * (size_t)i4;
    const float orientation = orc_orient2d(pa, pb, pc);
    float err;
    float det = orc_incircle_filter(pa, pb, pc, pd, &err);
    if (!((det > err) || (-det > err))) {
        (*n_exact)++;
        int swap = 0;
        uint32_t t;
        const float* v;
#define ORC_SW(x, y, px, py) { t = y; y = x; x = t; v = py; py = px; px = v; swap = !swap; }
        if (i1 > i3) ORC_SW(i1, i3, pa, pc);
        if (i2 > i4) ORC_SW(i2, i4, pb, pd);
        if (i1 > i2) ORC_SW(i1, i2, pa, pb);
        if (i3 > i4) ORC_SW(i3, i4, pc, pd);
        if (i2 > i3) ORC_SW(i2, i3, pb, pc);
#undef ORC_SW
        det = orc_incircle_exact(pa, pb, pc, pd);
        int depth = 0;
        while (det == 0.0f) {
            depth++;
            if (depth == 1) det = orc_orient2d(pb, pc, pd);
            else if (depth == 2) det = -orc_orient2d(pa, pc, pd);
            else det = ((swap + (orientation < 0.0f)) == 1) ? 1.0f : -1.0f;
        }
        if (swap) det = -det;
    }
    if (orientation < 0.0f) det = -det;
    return det;
}

int orc_ashape2d(uint32_t n, const float* coords, const float* alpha, orc_ashape2d_out* o) {
    memset(o, 0, sizeof *o);
    if (n < 2) return 1;
    o->n = n;
    // ---- LBVH over the 2D spheres (x, y, 0, r) -------------------------------
    float* s = (float*)malloc((size_t)n * 16);
    for (uint32_t i = 0; i < n; ++i) {
        s[4 * i] = coords[2 * i];
        s[4 * i + 1] = coords[2 * i + 1];
        s[4 * i + 2] = 0.0f;
        s[4 * i + 3] = alpha[i];
    }
    float bb[4];
    orc_bbox2d(n, s, bb);
    uint64_t* codes = (uint64_t*)malloc((size_t)n * 8);
    o->perm = (uint32_t*)malloc((size_t)n * 4);
    orc_morton2d(n, s, bb, codes);
    for (uint32_t i = 0; i < n; ++i) o->perm[i] = i;
    orc_sort_pairs(n, codes, o->perm);
    int32_t* sep = (int32_t*)malloc((size_t)n * 4);
    uint8_t* cil = (uint8_t*)malloc(n);
    uint32_t* lp = (uint32_t*)malloc((size_t)n * 4);
    uint32_t* ip = (uint32_t*)malloc((size_t)n * 4);
    orc_karras(n, codes, sep, cil, lp, ip);
    float* cm = (float*)malloc((size_t)(n + N_INF) * 16);
    for (uint32_t i = 0; i < n; ++i) memcpy(cm + 4 * i, s + 4 * (size_t)o->perm[i], 16);
    float* boxes = (float*)malloc((size_t)(n - 1) * 24);
    orc_fit(n, cm, sep, cil, 1, boxes);
    o->codes = codes;
    memcpy(o->bb_glob, bb, sizeof bb);
    // ---- infinity points (:144-166) ------------------------------------------
    {
        const float avg0 = 0.5f * (bb[2] + bb[0]), avg1 = 0.5f * (bb[3] + bb[1]);
        const float r0 = bb[2] - bb[0], r1 = bb[3] - bb[1];
        const float mr = fmaxf(r0, r1);
        const float m2 = 2.0f * mr;
        const float inf[3][2] = {{avg0 - m2, avg1 - m2}, {avg0 + m2, avg1 - m2}, {avg0, avg1 + m2}};
        for (int k = 0; k < 3; ++k) {
            float* p = cm + 4 * (size_t)(n + k);
            p[0] = inf[k][0];
            p[1] = inf[k][1];
            p[2] = 0.0f;
            p[3] = 0.0f;
        }
    }
    // ---- count pass and the per-node neighbour rows ----------------------------
    uint32_t* cnt = (uint32_t*)calloc(n, 4);
    uint32_t* roff = (uint32_t*)malloc(((size_t)n + 1) * 4);
    uint32_t err = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : err)
    for (long long t = 0; t < (long long)n; ++t) {
        uint32_t e = 0;
        cnt[t] = neighbours((uint32_t)t, cm, sep, cil, boxes, 0, NULL, &e);
        err |= e;
    }
    roff[0] = 0;
    for (uint32_t i = 0; i < n; ++i) roff[i + 1] = roff[i] + cnt[i];
    uint32_t* nb = (uint32_t*)malloc(((size_t)roff[n] + 1) * 4);
    o->nineig = (uint32_t*)malloc((size_t)n * 4);
    o->row_offset = roff;
    o->cand = nb;
    uint8_t* act = (uint8_t*)calloc((size_t)roff[n] + 1, 1);
    uint8_t* ntri_out = (uint8_t*)calloc(n, 1);
    uint32_t* nfneig = (uint32_t*)calloc(n, 4);
    o->nelem = (uint8_t*)calloc(n, 1);
    o->node_is_bnd = (uint8_t*)calloc(n, 1);
    uint32_t tmax = 0;
    for (uint32_t i = 0; i < n; ++i) tmax = cnt[i] + N_INF > tmax ? cnt[i] + N_INF : tmax;
    tri2* T_all = (tri2*)malloc((size_t)n * tmax * sizeof(tri2));
    uint32_t* tlast = (uint32_t*)calloc(n, 4);
    uint32_t n_exact = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(| : err) reduction(+ : n_exact)
    for (long long t = 0; t < (long long)n; ++t) {
        const uint32_t si = (uint32_t)t;
        uint32_t* row = nb + roff[si];
        uint32_t e = 0;
        const uint32_t k = neighbours(si, cm, sep, cil, boxes, 1, row, &e);
        err |= e;
        o->nineig[si] = k;
        tri2* T = T_all + (size_t)si * tmax;
        T[0] = (tri2){1, 2};
        T[1] = (tri2){2, 0};
        T[2] = (tri2){0, 1};
        uint32_t Tl = 3;
        if (k - N_INF < 2) {
            o->node_is_bnd[si] = 1;
            tlast[si] = 0;
            continue;
        }
        uint64_t tag[4];
        uint32_t ne = 0;
        for (uint32_t ni = N_INF; ni < k; ++ni) {
            tag[0] = tag[1] = tag[2] = tag[3] = 0;
            const uint32_t sj = gid(ni, n, row);
            uint32_t R = 0, ti = 0;
            while (ti < Tl) {
                const tri2 tr = T[ti];
                const float det = conflict2(cm, si, gid(tr.a, n, row), gid(tr.b, n, row), sj, &ne);
                if (det > 0.0f) {
                    tag[tr.a >> 6] ^= 1ULL << (tr.a & 63);
                    tag[tr.b >> 6] ^= 1ULL << (tr.b & 63);
                    R++;
                    Tl--;
                    T[ti] = T[Tl];
                } else {
                    ti++;
                }
            }
            if (R) {
                for (uint32_t j = 0; j < 4; ++j) {
                    const uint64_t v = tag[j];
                    const uint32_t end = (j + 1) * 64 > ni ? ni : (j + 1) * 64;
                    if (!v) continue;
                    for (uint32_t r = j * 64; r < end; ++r)
                        if (v & (1ULL << (r & 63))) {
                            if (Tl >= tmax) { e |= ORC_ERR_CAP; break; }
                            T[Tl++] = (tri2){(uint8_t)r, (uint8_t)ni};
                        }
                }
            }
        }
        n_exact += ne;
        // ---- filter (:528-595) ----
        tag[0] = tag[1] = tag[2] = tag[3] = 0;
        int bnd = 0;
        uint8_t nout = 0, nk = 0;
        uint32_t ti = 0;
        while (ti < Tl) {
            const tri2 tr = T[ti];
            if (tr.a < N_INF || tr.b < N_INF) {
                bnd = 1;
                Tl--;
                T[ti] = T[Tl];
                continue;
            }
            uint32_t i1 = si, i2 = gid(tr.a, n, row), i3 = gid(tr.b, n, row), tmp;
            int swap = 0;
            if (i3 < i2) { tmp = i3; i3 = i2; i2 = tmp; swap = !swap; }
            if (i2 < i1) { tmp = i2; i2 = i1; i1 = tmp; swap = !swap; }
            if (i3 < i2) { tmp = i3; i3 = i2; i2 = tmp; swap = !swap; }
            const float *p1 = cm + 4 * (size_t)i1, *p2 = cm + 4 * (size_t)i2, *p3 = cm + 4 * (size_t)i3;
            // (p3 - p2) x (p1 - p2)
            const float ux = p3[0] - p2[0], uy = p3[1] - p2[1], vx = p1[0] - p2[0], vy = p1[1] - p2[1];
            float det = ux * vy - uy * vx;
            if (swap) det = -det;
            const float l12 = sqn2(p1[0] - p2[0], p1[1] - p2[1]);
            const float l23 = sqn2(p2[0] - p3[0], p2[1] - p3[1]);
            const float l31 = sqn2(p3[0] - p1[0], p3[1] - p1[1]);
            const float crs = (l12 * l23 * l31) / (4.f * det * det);
            const float aeff = fminf(p3[3], fminf(p1[3], p2[3]));
            if (crs <= aeff * aeff) {
                tag[tr.a >> 6] |= 1ULL << (tr.a & 63);
                tag[tr.b >> 6] |= 1ULL << (tr.b & 63);
                act[roff[si] + tr.a - N_INF] += 1;
                act[roff[si] + tr.b - N_INF] += 1;
                nk++;
                if (det < 0) T[ti] = (tri2){tr.b, tr.a};
                ti++;
                nout += (si == i1);
            } else {
                bnd = 1;
                Tl--;
                T[ti] = T[Tl];
            }
        }
        tlast[si] = Tl;
        o->node_is_bnd[si] = (uint8_t)bnd;
        ntri_out[si] = nout;
        o->nelem[si] = nk;
        nfneig[si] = (uint32_t)(__builtin_popcountll(tag[0]) + __builtin_popcountll(tag[1]) +
                                __builtin_popcountll(tag[2]) + __builtin_popcountll(tag[3]));
        err |= e;
    }
    o->status = err;
    o->n_exact = n_exact;
    // ---- scans and compress (:602-690) ----------------------------------------
    o->elemrow = (uint32_t*)malloc(((size_t)n + 1) * 4);
    o->row = (uint32_t*)malloc(((size_t)n + 1) * 4);
    o->elemrow[0] = 0;
    o->row[0] = 0;
    for (uint32_t i = 0; i < n; ++i) {
        o->elemrow[i + 1] = o->elemrow[i] + ntri_out[i];
        o->row[i + 1] = o->row[i] + nfneig[i];
    }
    o->n_elems = o->elemrow[n];
    o->n_edges = o->row[n];
    o->elems = (uint32_t*)malloc(((size_t)o->n_elems + 1) * 12);
    o->neig = (uint32_t*)malloc(((size_t)o->n_edges + 1) * 4);
    o->edge_is_bnd = (uint8_t*)malloc((size_t)o->n_edges + 1);
#pragma omp parallel for schedule(dynamic, 256)
    for (long long t = 0; t < (long long)n; ++t) {
        const uint32_t si = (uint32_t)t;
        const uint32_t* row = nb + roff[si];
        uint32_t put = o->row[si];
        for (uint32_t i = N_INF; i < o->nineig[si]; ++i) {
            const uint8_t c = act[roff[si] + i - N_INF];
            if (c) {
                o->edge_is_bnd[put] = (c == 1);
                o->neig[put++] = gid(i, n, row);
            }
        }
        const tri2* T = T_all + (size_t)si * tmax;
        uint32_t idx = 0;
        for (uint32_t i = o->elemrow[si]; i < o->elemrow[si + 1]; ++i) {
            tri2 tc = T[idx];
            uint32_t a = gid(tc.a, n, row), b = gid(tc.b, n, row);
            while (a < si || b < si) {
                idx++;
                tc = T[idx];
                a = gid(tc.a, n, row);
                b = gid(tc.b, n, row);
            }
            o->elems[3 * (size_t)i] = si;
            o->elems[3 * (size_t)i + 1] = a;
            o->elems[3 * (size_t)i + 2] = b;
            idx++;
        }
    }
    o->coords_m = cm;
    free(s); free(sep); free(cil); free(lp); free(ip); free(boxes); free(cnt);
    free(act); free(ntri_out); free(nfneig); free(T_all); free(tlast);
    return 0;
}

void orc_ashape2d_free(orc_ashape2d_out* a) {
    free(a->perm); free(a->coords_m); free(a->nineig); free(a->cand); free(a->row_offset);
    free(a->elemrow); free(a->elems); free(a->row); free(a->neig); free(a->edge_is_bnd);
    free(a->node_is_bnd); free(a->nelem); free(a->codes);
    memset(a, 0, sizeof *a);
}
