// Oracle (test infrastructure only): plain-C restatement of the reference's
// Karras LBVH over 3D spheres, include/geometry/lbvh.hpp:141-360, with the
// Morton encoders of include/geometry/morton.hpp.  Sequential and
// deterministic; results are bit-identical to the reference's parallel build
// because every quantity it computes is order independent (min/max boxes,
// integer codes, stable sort).
#include "stream_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

// BBox<float,3>::empty() is (FLT_MAX, -FLT_MAX) (bbox.hpp:114-117, vec.hpp:246-259).
void orc_bbox3d(uint32_t n, const float* s, int use_radius, float out[6]) {
    float mn[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, mx[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    for (uint32_t i = 0; i < n; ++i) {
        const float r = use_radius ? s[4 * i + 3] : 0.0f;
        for (int k = 0; k < 3; ++k) {
            // Sphere::get_bbox: pmin -= r, pmax += r (primitives.hpp:136-141)
            float lo = use_radius ? s[4 * i + k] - r : s[4 * i + k];
            float hi = use_radius ? s[4 * i + k] + r : s[4 * i + k];
            mn[k] = fminf(mn[k], lo);
            mx[k] = fmaxf(mx[k], hi);
        }
    }
    for (int k = 0; k < 3; ++k) { out[k] = mn[k]; out[3 + k] = mx[k]; }
}

// splitBy3 / encode_magicbits3D (morton.hpp:27-45): 21 bits per axis.
static inline uint64_t spread21(uint32_t a) {
    uint64_t x = a & 0x1fffffu;
    x = (x | x << 32) & 0x1f00000000ffffULL;
    x = (x | x << 16) & 0x1f0000ff0000ffULL;
    x = (x | x << 8) & 0x100f00f00f00f00fULL;
    x = (x | x << 4) & 0x10c30c30c30c30c3ULL;
    x = (x | x << 2) & 0x1249249249249249ULL;
    return x;
}
// splitBy3_32 / encode_magicbits3D_32 (morton.hpp:47-59): 10 bits per axis.
static inline uint32_t spread10(uint32_t a) {
    uint32_t x = a & 0x3ffu;
    x = (x | x << 16) & 0x30000ffu;
    x = (x | x << 8) & 0x0300f00fu;
    x = (x | x << 4) & 0x30c30c3u;
    x = (x | x << 2) & 0x9249249u;
    return x;
}
// static_cast<uint32_t>(float) for the quantised coordinate; a NaN (zero
// extent) maps to 0 as on both host and device.
static inline uint32_t f2u(float c) {
    if (!(c >= 0.0f)) return 0u;
    if (c >= 4294967296.0f) return 0u;
    return (uint32_t)c;
}

// _compute_morton_codes (lbvh.hpp:178-213).
void orc_morton3d(uint32_t n, const float* s, const float bb[6], int bits, uint64_t* codes) {
    const float imax = (bits == 30) ? 1024.0f : 2097152.0f;  // 2^(bits/3)
    float f[3];
    for (int k = 0; k < 3; ++k) {
        float range = bb[3 + k] - bb[k];
        float fk = imax / range;
        if (range * fk >= imax) fk = nextafterf(fk, 0.0f);
        f[k] = fk;
    }
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t q[3];
        for (int k = 0; k < 3; ++k) q[k] = f2u((s[4 * i + k] - bb[k]) * f[k]);
        if (bits == 30)
            codes[i] = (uint64_t)(spread10(q[0]) | (spread10(q[1]) << 1) | (spread10(q[2]) << 2));
        else
            codes[i] = spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
    }
}

// Stable LSD radix sort, 8-bit digits, skipping digit positions on which all
// keys agree (a stable pass over a constant digit is the identity).
void orc_sort_pairs(uint32_t n, uint64_t* keys, uint32_t* vals) {
    uint64_t* k2 = (uint64_t*)malloc((size_t)n * 8);
    uint32_t* v2 = (uint32_t*)malloc((size_t)n * 4);
    uint64_t *ki = keys, *ko = k2;
    uint32_t *vi = vals, *vo = v2;
    for (int pass = 0; pass < 8; ++pass) {
        size_t cnt[257];
        memset(cnt, 0, sizeof cnt);
        const int sh = 8 * pass;
        for (uint32_t i = 0; i < n; ++i) cnt[((ki[i] >> sh) & 0xff) + 1]++;
        int trivial = 0;
        for (int d = 0; d < 256; ++d) if (cnt[d + 1] == n) trivial = 1;
        if (trivial) continue;
        for (int d = 0; d < 256; ++d) cnt[d + 1] += cnt[d];
        for (uint32_t i = 0; i < n; ++i) {
            size_t p = cnt[(ki[i] >> sh) & 0xff]++;
            ko[p] = ki[i];
            vo[p] = vi[i];
        }
        uint64_t* tk = ki; ki = ko; ko = tk;
        uint32_t* tv = vi; vi = vo; vo = tv;
    }
    if (ki != keys) {
        memcpy(keys, ki, (size_t)n * 8);
        memcpy(vals, vi, (size_t)n * 4);
    }
    free(k2);
    free(v2);
}

// _build_hierarchy (lbvh.hpp:246-308).
void orc_karras(uint32_t n32, const uint64_t* m, int32_t* sep, uint8_t* cil, uint32_t* leaf_parent,
                uint32_t* internal_parent) {
    const int n = (int)n32;
    for (int i = 0; i < n - 1; ++i) {
        const uint64_t mi = m[i];
        const int dp1 = (i + 1 >= n) ? -1 : clz64(mi ^ m[i + 1]);
        const int dm1 = (i - 1 < 0) ? -1 : clz64(mi ^ m[i - 1]);
        const int d = (dp1 - dm1 > 0) ? 1 : -1;
        const int dmin = (i - d < n && i - d >= 0) ? clz64(mi ^ m[i - d]) : -1;
        int lmax = 2;
        while (i + lmax * d >= 0 && i + lmax * d < n && clz64(mi ^ m[i + lmax * d]) > dmin) lmax *= 2;
        int l = 0;
        for (int t = lmax / 2; t >= 1; t /= 2) {
            const int k = i + (l + t) * d;
            if (k >= 0 && k < n && clz64(mi ^ m[k]) > dmin) l += t;
        }
        const int j = i + l * d;
        int gamma = (i + j) >> 1;
        const uint64_t mj = m[j];
        if (mi != mj) {
            const int dnode = clz64(mi ^ mj);
            int s = 0;
            for (int t = (l + 1) / 2; t >= 1; t = (t + 1) / 2) {
                const int k = i + (s + t) * d;
                if (k >= 0 && k < n && clz64(mi ^ m[k]) > dnode) s += t;
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
}

static inline void leaf_box(const float* o, int fit_point, float b[6]) {
    for (int k = 0; k < 3; ++k) {
        b[k] = fit_point ? o[k] : o[k] - o[3];
        b[3 + k] = fit_point ? o[k] : o[k] + o[3];
    }
}
static inline void combine(float* a, const float* b) {
    for (int k = 0; k < 3; ++k) a[k] = fminf(a[k], b[k]);
    for (int k = 0; k < 3; ++k) a[3 + k] = fmaxf(a[3 + k], b[3 + k]);
}

// fit (lbvh.hpp:311-351): the same "second arrival continues" protocol, run
// leaf by leaf.  Box union is exact and commutative, so the order of arrival
// does not change the result.
void orc_fit(uint32_t n, const float* obj_m, const int32_t* sep, const uint8_t* cil,
             int fit_point, float* bboxes) {
    // parents are recomputed from sep/cil to keep the signature small
    uint32_t* lp = (uint32_t*)malloc((size_t)n * 4);
    uint32_t* ip = (uint32_t*)malloc((size_t)n * 4);
    uint8_t* touched = (uint8_t*)calloc(n, 1);
    for (uint32_t i = 0; i + 1 < n; ++i) {
        const int g = sep[i];
        if (cil[i] & 1) lp[g] = i; else ip[g] = i;
        if (cil[i] & 2) lp[g + 1] = i | 0x80000000u; else ip[g + 1] = i | 0x80000000u;
    }
    ip[0] = n;
    for (uint32_t i = 0; i < n; ++i) {
        float data[6];
        leaf_box(obj_m + 4 * i, fit_point, data);
        uint32_t p = lp[i];
        int right = (p & 0x80000000u) != 0;
        p &= 0x7fffffffu;
        while (p < n) {
            const uint8_t old = touched[p];
            touched[p] = 1;
            if (!old) break;
            const uint32_t other = (uint32_t)sep[p] + (uint32_t)(!right);
            float ob[6];
            if (cil[p] & ((!right) + 1)) leaf_box(obj_m + 4 * other, fit_point, ob);
            else memcpy(ob, bboxes + 6 * (size_t)other, sizeof ob);
            combine(data, ob);
            memcpy(bboxes + 6 * (size_t)p, data, sizeof data);
            const uint32_t pp = ip[p];
            right = (pp & 0x80000000u) != 0;
            p = pp & 0x7fffffffu;
        }
    }
    free(lp);
    free(ip);
    free(touched);
}

int orc_lbvh3d(uint32_t n, const float* s, int bits, int fit_point, float* bb_glob,
               uint64_t* codes_sorted, uint32_t* perm, int32_t* sep, uint8_t* cil,
               uint32_t* leaf_parent, uint32_t* internal_parent, float* bboxes, float* obj_m) {
    if (n < 2) return 1;
    float bb[6];
    orc_bbox3d(n, s, 1, bb);
    uint64_t* codes = (uint64_t*)malloc((size_t)n * 8);
    uint32_t* map = (uint32_t*)malloc((size_t)n * 4);
    orc_morton3d(n, s, bb, bits, codes);
    for (uint32_t i = 0; i < n; ++i) map[i] = i;
    orc_sort_pairs(n, codes, map);
    int32_t* sp = (int32_t*)malloc((size_t)n * 4);
    uint8_t* cl = (uint8_t*)malloc(n);
    uint32_t* lp = (uint32_t*)malloc((size_t)n * 4);
    uint32_t* ip = (uint32_t*)malloc((size_t)n * 4);
    orc_karras(n, codes, sp, cl, lp, ip);
    float* om = (float*)malloc((size_t)n * 16);
    for (uint32_t i = 0; i < n; ++i) memcpy(om + 4 * i, s + 4 * (size_t)map[i], 16);
    float* bx = (float*)malloc((size_t)(n - 1) * 24);
    orc_fit(n, om, sp, cl, fit_point, bx);
    if (bb_glob) memcpy(bb_glob, bb, sizeof bb);
    if (codes_sorted) memcpy(codes_sorted, codes, (size_t)n * 8);
    if (perm) memcpy(perm, map, (size_t)n * 4);
    if (sep) memcpy(sep, sp, (size_t)(n - 1) * 4);
    if (cil) memcpy(cil, cl, n - 1);
    if (leaf_parent) memcpy(leaf_parent, lp, (size_t)n * 4);
    if (internal_parent) memcpy(internal_parent, ip, (size_t)(n - 1) * 4);
    if (bboxes) memcpy(bboxes, bx, (size_t)(n - 1) * 24);
    if (obj_m) memcpy(obj_m, om, (size_t)n * 16);
    free(codes); free(map); free(sp); free(cl); free(lp); free(ip); free(om); free(bx);
    return 0;
}

// ---- 2D (LBVH<Sphere2D, ..., 2>) ------------------------------------------
// Global box of 2D spheres, radius included: out = pmin[2], pmax[2].
// s holds n x 4 floats (x, y, unused, r).
void orc_bbox2d(uint32_t n, const float* s, float out[4]) {
    float mn[2] = {FLT_MAX, FLT_MAX}, mx[2] = {-FLT_MAX, -FLT_MAX};
    for (uint32_t i = 0; i < n; ++i) {
        const float r = s[4 * i + 3];
        for (int k = 0; k < 2; ++k) {
            mn[k] = fminf(mn[k], s[4 * i + k] - r);
            mx[k] = fmaxf(mx[k], s[4 * i + k] + r);
        }
    }
    out[0] = mn[0]; out[1] = mn[1]; out[2] = mx[0]; out[3] = mx[1];
}

// splitBy2 / encode_magicbits2D (morton.hpp:61-76): 32 bits per axis.
static inline uint64_t spread32(uint32_t a) {
    uint64_t x = a;
    x = (x | x << 16) & 0x0000FFFF0000FFFFULL;
    x = (x | x << 8) & 0x00FF00FF00FF00FFULL;
    x = (x | x << 4) & 0x0F0F0F0F0F0F0F0FULL;
    x = (x | x << 2) & 0x3333333333333333ULL;
    x = (x | x << 1) & 0x5555555555555555ULL;
    return x;
}

// _compute_morton_codes with dim = 2 (lbvh.hpp:178-213): imax = 2^32.
void orc_morton2d(uint32_t n, const float* s, const float bb[4], uint64_t* codes) {
    const float imax = 4294967296.0f;
    float f[2];
    for (int k = 0; k < 2; ++k) {
        const float range = bb[2 + k] - bb[k];
        float fk = imax / range;
        if (range * fk >= imax) fk = nextafterf(fk, 0.0f);
        f[k] = fk;
    }
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t qx = f2u((s[4 * i] - bb[0]) * f[0]);
        const uint32_t qy = f2u((s[4 * i + 1] - bb[1]) * f[1]);
        codes[i] = spread32(qx) | (spread32(qy) << 1);
    }
}
