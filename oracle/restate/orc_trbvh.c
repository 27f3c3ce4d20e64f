// Oracle (test infrastructure only): plain-C restatement of the TRBVH of
// include/geometry/trbvh.hpp: Apetrei agglomerative build (:245-390) and
// Karras-Aila treelet restructuring (:392-633, 3 rounds at :666-674).
//
// Node ids: leaves 0..n-1 (Morton order), internal nodes n..2n-2; the root's
// parent is 2n.  The build topology, boxes and subtree sizes are
// deterministic and equal to the reference's.  The reference's SAH values are
// not: a thread's running cost starts from its own leaf's area while sibling
// leaves count 0 (:326-327,371-373), so they depend on which child arrives
// second.  This restatement (and the GPU) use the order-independent SAH
// cost(leaf) = Ct A(leaf), cost(node) = (Ci A(node) + cost(left)) + cost(right),
// which makes the restructured tree a deterministic function of the input.
// Where every leaf box has zero area (spheres of radius 0) the two
// definitions agree: the reference's running cost then starts from 0, and a
// thread that runs the leaves in index order reaches every parent from its
// right child, so its sums are cost(right) + (Ci A + cost(left)).  Ci A(node)
// is formed as (Ci * ext_x) * ext_y in the 2D measure, the reference's
// association (:373).
// Treelet size and the area measure are parameters: the reference fixes 5
// leaves and the 2D product ext_x * ext_y (:74,328,373,471); the 3D
// half-surface xy + yz + zx is the natural 3D measure.
#include "stream_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define TR_CI 1.2f
#define TR_CT 1.0f
#define TR_MAXK 8

static inline float area_of(const float* b, int area3d) {
    const float ex = b[3] - b[0], ey = b[4] - b[1], ez = b[5] - b[2];
    return area3d ? (ex * ey + ey * ez) + ez * ex : ex * ey;
}
// Ci * A(node) of the Apetrei build: the reference multiplies left to right,
// (Ci * ext_x) * ext_y (trbvh.hpp:373); the 3D measure has no reference.
static inline float ci_area_of(const float* b, int area3d) {
    const float ex = b[3] - b[0], ey = b[4] - b[1];
    return area3d ? TR_CI * area_of(b, 1) : (TR_CI * ex) * ey;
}
static inline void box_union(float* a, const float* b) {
    for (int k = 0; k < 3; ++k) a[k] = fminf(a[k], b[k]);
    for (int k = 0; k < 3; ++k) a[3 + k] = fmaxf(a[3 + k], b[3 + k]);
}

// Apetrei bottom-up build (trbvh.hpp:299-390), one leaf after the other with
// the same "second arrival continues" rule.
static void apetrei(uint32_t n, const uint64_t* codes, const float* obj_m, int area3d, orc_trbvh* t) {
    uint64_t* delta = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n - 1 : 1));
    for (uint32_t i = 0; i + 1 < n; ++i) delta[i] = codes[i] ^ codes[i + 1];
    uint32_t* touched = (uint32_t*)calloc(n, 4);
    for (uint32_t i = 0; i < n; ++i) {
        float* b = t->bboxes + 6 * (size_t)i;
        const float* o = obj_m + 4 * (size_t)i;
        for (int k = 0; k < 3; ++k) { b[k] = o[k] - o[3]; b[3 + k] = o[k] + o[3]; }
        t->subtree_size[i] = 1;
        t->sah[i] = TR_CT * area_of(b, area3d);
    }
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t idx = i, imin = i, imax = i;
        for (;;) {
            if (imin == 0 && imax == n - 1) {
                t->parent[idx] = 2 * n;
                t->root = idx;
                break;
            }
            const int right_parent = imin == 0 || (imax != n - 1 && delta[imax] < delta[imin - 1]);
            uint32_t parent;
            if (right_parent) {
                parent = imax + n;
                t->child_left[parent - n] = idx;
                t->range_min[parent - n] = imin;
            } else {
                parent = imin + n - 1;
                t->child_right[parent - n] = idx;
                t->range_max[parent - n] = imax;
            }
            t->parent[idx] = parent;
            if (touched[parent - n]++ == 0) break;
            const uint32_t l = t->child_left[parent - n], r = t->child_right[parent - n];
            float* pb = t->bboxes + 6 * (size_t)parent;
            memcpy(pb, t->bboxes + 6 * (size_t)l, 24);
            box_union(pb, t->bboxes + 6 * (size_t)r);
            t->subtree_size[parent] = t->subtree_size[l] + t->subtree_size[r];
            t->sah[parent] = (ci_area_of(pb, area3d) + t->sah[l]) + t->sah[r];
            idx = parent;
            if (right_parent) imax = t->range_max[parent - n];
            else imin = t->range_min[parent - n];
        }
    }
    free(delta);
    free(touched);
}

// One treelet restructuring rooted at internal node idx (trbvh.hpp:407-618),
// growing the treelet by the internal leaf of largest cost.
static void treelet(uint32_t n, uint32_t idx, int K, int area3d, orc_trbvh* t) {
    uint32_t inner[TR_MAXK], leaves[TR_MAXK];
    float cost[TR_MAXK];
    inner[0] = idx;
    leaves[0] = t->child_left[idx - n];
    leaves[1] = t->child_right[idx - n];
    cost[0] = t->sah[leaves[0]];
    cost[1] = t->sah[leaves[1]];
    for (int in = 1; in < K - 1; ++in) {
        int best = -1;
        float bc = -FLT_MAX;
        for (int l = 0; l <= in; ++l)
            if (leaves[l] >= n && (best < 0 || cost[l] > bc)) { bc = cost[l]; best = l; }
        if (best < 0) return;  // fewer internal nodes than the treelet needs
        const uint32_t bl = leaves[best];
        inner[in] = bl;
        leaves[best] = leaves[in];
        cost[best] = cost[in];
        leaves[in] = t->child_left[bl - n];
        cost[in] = t->sah[leaves[in]];
        leaves[in + 1] = t->child_right[bl - n];
        cost[in + 1] = t->sah[leaves[in + 1]];
    }
    const int ns = 1 << K, mask = ns - 1;
    float areas[1 << TR_MAXK], copt[1 << TR_MAXK];
    uint8_t popt[1 << TR_MAXK];
    uint32_t tsz[1 << TR_MAXK];
    for (int s = 1; s < ns; ++s) {
        float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
        uint32_t sz = 0;
        for (int l = 0; l < K; ++l)
            if (s & (1 << l)) { box_union(b, t->bboxes + 6 * (size_t)leaves[l]); sz += t->subtree_size[leaves[l]]; }
        areas[s] = area_of(b, area3d);
        tsz[s] = sz;
        copt[s] = 0.0f;
        popt[s] = 0;
    }
    for (int l = 0; l < K; ++l) copt[1 << l] = cost[l];
    for (int k = 2; k <= K; ++k) {
        for (int s = 1; s < ns; ++s) {
            if (__builtin_popcount((unsigned)s) != k) continue;
            float cs = FLT_MAX;
            int ps = 0;
            const int delta = (s - 1) & s;
            int p = (-delta) & s;
            while (p != 0) {
                const float c = copt[p] + copt[s ^ p];
                if (c < cs) { cs = c; ps = p; }
                p = (p - delta) & s;
            }
            copt[s] = fminf(TR_CI * areas[s] + cs, TR_CT * areas[s] * (float)tsz[s]);
            popt[s] = (uint8_t)ps;
        }
    }
    // Rebuild (trbvh.hpp:525-618): LIFO over partitions; a partition pushed as
    // "left" becomes the right child, as in the reference.
    int index = 0;
    uint8_t stp[2 * TR_MAXK], stl[2 * TR_MAXK];
    uint32_t stpar[2 * TR_MAXK];
    int ss = 0;
    t->sah[idx] = copt[mask];
    stp[ss] = popt[mask]; stl[ss] = 1; stpar[ss] = inner[0]; ++ss;
    stp[ss] = (uint8_t)((~popt[mask]) & mask); stl[ss] = 0; stpar[ss] = inner[0]; ++ss;
    while (ss) {
        --ss;
        const int part = stp[ss], isl = stl[ss];
        const uint32_t par = stpar[ss];
        const int leaf = __builtin_popcount((unsigned)part) == 1;
        const uint32_t node = leaf ? leaves[__builtin_ffs(part) - 1] : inner[++index];
        if (isl) t->child_right[par - n] = node;
        else t->child_left[par - n] = node;
        t->parent[node] = par;
        if (!leaf) {
            float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
            for (int l = 0; l < K; ++l)
                if (part & (1 << l)) box_union(b, t->bboxes + 6 * (size_t)leaves[l]);
            memcpy(t->bboxes + 6 * (size_t)node, b, 24);
            t->subtree_size[node] = tsz[part];
            t->sah[node] = copt[part];
            const int pl = popt[part], pr = (~pl) & part;
            stp[ss] = (uint8_t)pl; stl[ss] = 1; stpar[ss] = node; ++ss;
            stp[ss] = (uint8_t)pr; stl[ss] = 0; stpar[ss] = node; ++ss;
        }
    }
}

// Post-order of the internal nodes of the current tree.
static uint32_t post_order(uint32_t n, const orc_trbvh* t, uint32_t* out) {
    uint32_t* st = (uint32_t*)malloc(sizeof(uint32_t) * 2 * n);
    uint8_t* vis = (uint8_t*)calloc(n, 1);
    uint32_t ss = 0, m = 0;
    st[ss++] = t->root;
    while (ss) {
        const uint32_t x = st[ss - 1];
        const uint32_t l = t->child_left[x - n], r = t->child_right[x - n];
        if (!vis[x - n]) {
            vis[x - n] = 1;
            if (r >= n) st[ss++] = r;
            if (l >= n) st[ss++] = l;
        } else {
            out[m++] = x;
            --ss;
        }
    }
    free(st);
    free(vis);
    return m;
}

int orc_trbvh3d(uint32_t n, const float* xyzr, int treelet_size, int area3d, int rounds, orc_trbvh* t) {
    if (n < 2 || treelet_size < 3 || treelet_size > TR_MAXK) return 1;
    memset(t, 0, sizeof *t);
    t->n = n;
    const size_t m = 2 * (size_t)n - 1;
    t->child_left = (uint32_t*)calloc(n - 1, 4);
    t->child_right = (uint32_t*)calloc(n - 1, 4);
    t->range_min = (uint32_t*)calloc(n - 1, 4);
    t->range_max = (uint32_t*)calloc(n - 1, 4);
    t->parent = (uint32_t*)calloc(m, 4);
    t->bboxes = (float*)calloc(m * 6, 4);
    t->subtree_size = (uint32_t*)calloc(m, 4);
    t->sah = (float*)calloc(m, 4);
    t->obj_m = (float*)malloc((size_t)n * 16);
    uint64_t* codes = (uint64_t*)malloc((size_t)n * 8);
    orc_lbvh3d(n, xyzr, 63, 0, NULL, codes, NULL, NULL, NULL, NULL, NULL, NULL, t->obj_m);
    apetrei(n, codes, t->obj_m, area3d, t);
    free(codes);
    uint32_t* order = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t min_size = (uint32_t)treelet_size;
    for (int r = 0; r < rounds; ++r) {
        const uint32_t cnt = post_order(n, t, order);
        for (uint32_t k = 0; k < cnt; ++k)
            if (t->subtree_size[order[k]] >= min_size) treelet(n, order[k], treelet_size, area3d, t);
        min_size *= 2;
    }
    free(order);
    return 0;
}

void orc_trbvh3d_free(orc_trbvh* t) {
    free(t->child_left); free(t->child_right); free(t->range_min); free(t->range_max); free(t->parent);
    free(t->bboxes); free(t->subtree_size); free(t->sah); free(t->obj_m);
    memset(t, 0, sizeof *t);
}

// Number of ordered pairs (i, j), i != j, of overlapping spheres found by a
// depth-first search of the tree (the query of
// tests/geometry/trbvh_random_collision.cpp, in 3D); out[i] per sphere.
void orc_trbvh3d_count(const orc_trbvh* t, uint32_t* out) {
    const uint32_t n = t->n;
    for (uint32_t q = 0; q < n; ++q) {
        uint32_t st[128], ss = 0, c = 0;
        st[ss++] = t->root;
        const float* s = t->obj_m + 4 * (size_t)q;
        while (ss) {
            const uint32_t cur = st[--ss];
            const uint32_t ch[2] = {t->child_left[cur - n], t->child_right[cur - n]};
            for (int k = 0; k < 2; ++k) {
                const uint32_t x = ch[k];
                if (x >= n) {
                    const float* b = t->bboxes + 6 * (size_t)x;
                    int in = 1;
                    for (int d = 0; d < 3; ++d) {
                        in &= s[d] - s[3] < b[3 + d];
                        in &= s[d] + s[3] > b[d];
                    }
                    if (in && ss < 128) st[ss++] = x;
                } else if (x != q) {
                    const float* o = t->obj_m + 4 * (size_t)x;
                    const float rs = s[3] + o[3];
                    const float dx = s[0] - o[0], dy = s[1] - o[1], dz = s[2] - o[2];
                    if (dx * dx + dy * dy + dz * dz <= rs * rs) ++c;
                }
            }
        }
        out[q] = c;
    }
}
