// Oracle (test infrastructure only): plain-C restatement of the reference's
// FP32 geometric predicates, include/geometry/predicates.hpp.
//
// The reference evaluates Shewchuk's adaptive predicates entirely in FP32
// (fp_tt = float, include/defines.h:24; splitter 4097 and epsilon 2^-24 at
// predicates.hpp:26-27).  Bit-exact parity with it (including its behaviour
// when an FP32 expansion tail underflows) requires the same sequence of IEEE
// operations, so every error-free transformation below performs the same
// float operations, in the same order, as the macro it restates
// (predicates.hpp:29-227).  Compile with -ffp-contract=off; the explicit
// fmaf() calls of the filter (predicates.hpp:1041-1097) stay fused.
#include "stream_oracle.h"

#include <math.h>

#define ORC_SPLITTER 4097.0f
#define ORC_EPS 5.9604644775390625e-08f
// predicates.hpp:588-589, computed in double from the float epsilon and then
// rounded to float, as the reference's constexpr initialisers are.
static const float k_isperrboundA = (float)((16.0 + 224.0 * (double)ORC_EPS) * (double)ORC_EPS);
static const float k_o3derrboundA = (float)((7.0 + 56.0 * (double)ORC_EPS) * (double)ORC_EPS);

// ---- error-free transformations (predicates.hpp:29-88) -------------------
static inline void two_sum(float a, float b, float* x, float* y) {
    float s = a + b;
    float bv = s - a;
    float av = s - bv;
    float br = b - bv;
    float ar = a - av;
    *x = s;
    *y = ar + br;
}
static inline void fast_two_sum(float a, float b, float* x, float* y) {
    float s = a + b;
    float bv = s - a;
    *x = s;
    *y = b - bv;
}
static inline void two_diff(float a, float b, float* x, float* y) {
    float d = a - b;
    float bv = a - d;
    float av = d + bv;
    float br = bv - b;
    float ar = a - av;
    *x = d;
    *y = ar + br;
}
static inline void split(float a, float* hi, float* lo) {
    float c = ORC_SPLITTER * a;
    float big = c - a;
    *hi = c - big;
    *lo = a - *hi;
}
// Two_Product_Presplit: b already split into (bhi, blo); a is split here.
static inline void two_product_presplit(float a, float b, float bhi, float blo, float* x, float* y) {
    float p = a * b;
    float ahi, alo;
    split(a, &ahi, &alo);
    float e1 = p - (ahi * bhi);
    float e2 = e1 - (alo * bhi);
    float e3 = e2 - (ahi * blo);
    *x = p;
    *y = (alo * blo) - e3;
}
static inline void two_product(float a, float b, float* x, float* y) {
    // Two_Product splits a before b; both splits are pure, so the result is
    // the same as splitting b first.
    float bhi, blo;
    float p = a * b;
    float ahi, alo;
    split(a, &ahi, &alo);
    split(b, &bhi, &blo);
    float e1 = p - (ahi * bhi);
    float e2 = e1 - (alo * bhi);
    float e3 = e2 - (ahi * blo);
    *x = p;
    *y = (alo * blo) - e3;
}
// Two_Two_Diff (predicates.hpp:124-126 via Two_One_Diff 116-118):
// (a1 + a0) - (b1 + b0) as a 4-component expansion x[0..3] (x[0] smallest).
static inline void two_two_diff(float a1, float a0, float b1, float b0, float x[4]) {
    float i, j, z;
    // Two_One_Diff(a1, a0, b0) -> (j, z, x0)
    two_diff(a0, b0, &i, &x[0]);
    two_sum(a1, i, &j, &z);
    // Two_One_Diff(j, z, b1) -> (x3, x2, x1)
    two_diff(z, b1, &i, &x[1]);
    two_sum(j, i, &x[3], &x[2]);
}
// 2x2 minor p_x * q_y - q_x * p_y as an expansion (the 'ab', 'bc', ... blocks
// of orient3dexact / insphereexact).
static inline void minor2(const float* p, const float* q, float m[4]) {
    float h1, l1, h2, l2;
    two_product(p[0], q[1], &h1, &l1);
    two_product(q[0], p[1], &h2, &l2);
    two_two_diff(h1, l1, h2, l2, m);
}

// fast_expansion_sum_zeroelim (predicates.hpp:229-296).  h must not alias.
static int fes_zeroelim(int elen, const float* e, int flen, const float* f, float* h) {
    float Q, Qn, hh;
    int ei = 0, fi = 0, hi = 0;
    float en = e[0], fn = f[0];
#define ORC_NEXT_E() (en = (++ei < elen) ? e[ei] : 0.0f)
#define ORC_NEXT_F() (fn = (++fi < flen) ? f[fi] : 0.0f)
    if ((fn > en) == (fn > -en)) { Q = en; ORC_NEXT_E(); }
    else { Q = fn; ORC_NEXT_F(); }
    if (ei < elen && fi < flen) {
        if ((fn > en) == (fn > -en)) { fast_two_sum(en, Q, &Qn, &hh); ORC_NEXT_E(); }
        else { fast_two_sum(fn, Q, &Qn, &hh); ORC_NEXT_F(); }
        Q = Qn;
        if (hh != 0.0f) h[hi++] = hh;
        while (ei < elen && fi < flen) {
            if ((fn > en) == (fn > -en)) { two_sum(Q, en, &Qn, &hh); ORC_NEXT_E(); }
            else { two_sum(Q, fn, &Qn, &hh); ORC_NEXT_F(); }
            Q = Qn;
            if (hh != 0.0f) h[hi++] = hh;
        }
    }
    while (ei < elen) {
        two_sum(Q, en, &Qn, &hh);
        ORC_NEXT_E();
        Q = Qn;
        if (hh != 0.0f) h[hi++] = hh;
    }
    while (fi < flen) {
        two_sum(Q, fn, &Qn, &hh);
        ORC_NEXT_F();
        Q = Qn;
        if (hh != 0.0f) h[hi++] = hh;
    }
#undef ORC_NEXT_E
#undef ORC_NEXT_F
    if (Q != 0.0f || hi == 0) h[hi++] = Q;
    return hi;
}

// scale_expansion_zeroelim (predicates.hpp:298-335).
static int se_zeroelim(int elen, const float* e, float b, float* h) {
    float bhi, blo, Q, hh, p1, p0, s;
    split(b, &bhi, &blo);
    two_product_presplit(e[0], b, bhi, blo, &Q, &hh);
    int hi = 0;
    if (hh != 0.0f) h[hi++] = hh;
    for (int i = 1; i < elen; ++i) {
        two_product_presplit(e[i], b, bhi, blo, &p1, &p0);
        two_sum(Q, p0, &s, &hh);
        if (hh != 0.0f) h[hi++] = hh;
        fast_two_sum(p1, s, &Q, &hh);
        if (hh != 0.0f) h[hi++] = hh;
    }
    if (Q != 0.0f || hi == 0) h[hi++] = Q;
    return hi;
}

// orient3dexact (predicates.hpp:591-670).
float orc_orient3d_exact(const float* pa, const float* pb, const float* pc, const float* pd) {
    float ab[4], bc[4], cd[4], da[4], ac[4], bd[4];
    float t8[8], abc[12], bcd[12], cda[12], dab[12];
    float adet[24], bdet[24], cdet[24], ddet[24], abdet[48], cddet[48], det[96];
    minor2(pa, pb, ab);
    minor2(pb, pc, bc);
    minor2(pc, pd, cd);
    minor2(pd, pa, da);
    minor2(pa, pc, ac);
    minor2(pb, pd, bd);
    int tl = fes_zeroelim(4, cd, 4, da, t8);
    int cdal = fes_zeroelim(tl, t8, 4, ac, cda);
    tl = fes_zeroelim(4, da, 4, ab, t8);
    int dabl = fes_zeroelim(tl, t8, 4, bd, dab);
    for (int i = 0; i < 4; ++i) { bd[i] = -bd[i]; ac[i] = -ac[i]; }
    tl = fes_zeroelim(4, ab, 4, bc, t8);
    int abcl = fes_zeroelim(tl, t8, 4, ac, abc);
    tl = fes_zeroelim(4, bc, 4, cd, t8);
    int bcdl = fes_zeroelim(tl, t8, 4, bd, bcd);
    int al = se_zeroelim(bcdl, bcd, pa[2], adet);
    int bl = se_zeroelim(cdal, cda, -pb[2], bdet);
    int cl = se_zeroelim(dabl, dab, pc[2], cdet);
    int dl = se_zeroelim(abcl, abc, -pd[2], ddet);
    int abl = fes_zeroelim(al, adet, bl, bdet, abdet);
    int cdl = fes_zeroelim(cl, cdet, dl, ddet, cddet);
    int n = fes_zeroelim(abl, abdet, cdl, cddet, det);
    return det[n - 1];
}

// orient3d: FP32 filter then exact (predicates.hpp:671-714).
float orc_orient3d(const float* pa, const float* pb, const float* pc, const float* pd) {
    float adx = pa[0] - pd[0], bdx = pb[0] - pd[0], cdx = pc[0] - pd[0];
    float ady = pa[1] - pd[1], bdy = pb[1] - pd[1], cdy = pc[1] - pd[1];
    float adz = pa[2] - pd[2], bdz = pb[2] - pd[2], cdz = pc[2] - pd[2];
    float bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    float cdxady = cdx * ady, adxcdy = adx * cdy;
    float adxbdy = adx * bdy, bdxady = bdx * ady;
    float det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
    float perm = (fabsf(bdxcdy) + fabsf(cdxbdy)) * fabsf(adz) +
                 (fabsf(cdxady) + fabsf(adxcdy)) * fabsf(bdz) +
                 (fabsf(adxbdy) + fabsf(bdxady)) * fabsf(cdz);
    float eb = k_o3derrboundA * perm;
    if (det > eb || -det > eb) return det;
    return orc_orient3d_exact(pa, pb, pc, pd);
}

// 3x3 minor of the lifted insphere matrix: s3*M3 + (s1*M1 + s2*M2), the
// abc/bcd/... blocks of insphereexact (predicates.hpp:818-876).
static int minor3(const float* m1, float s1, const float* m2, float s2, const float* m3, float s3,
                  float* out) {
    float t8a[8], t8b[8], t16[16];
    int la = se_zeroelim(4, m1, s1, t8a);
    int lb = se_zeroelim(4, m2, s2, t8b);
    int l16 = fes_zeroelim(la, t8a, lb, t8b, t16);
    la = se_zeroelim(4, m3, s3, t8a);
    return fes_zeroelim(la, t8a, l16, t16, out);
}
// (p + q) - (r + s) for 3x3 minors (the bcde/cdea/... blocks, predicates.hpp:878-956).
static int minor4(const float* p, int lp, const float* q, int lq, const float* r, int lr,
                  const float* s, int ls, float* out) {
    float a[48], b[48];
    int la = fes_zeroelim(lp, p, lq, q, a);
    int lb = fes_zeroelim(lr, r, ls, s, b);
    for (int i = 0; i < lb; ++i) b[i] = -b[i];
    return fes_zeroelim(la, a, lb, b, out);
}
// minor * (px^2 + py^2 + pz^2) as an expansion (the '*lift' blocks).
static int lift(const float* m, int lm, const float* p, float* out) {
    float t192[192], x[384], y[384], z[384], xy[768];
    int l = se_zeroelim(lm, m, p[0], t192);
    int lx = se_zeroelim(l, t192, p[0], x);
    l = se_zeroelim(lm, m, p[1], t192);
    int ly = se_zeroelim(l, t192, p[1], y);
    l = se_zeroelim(lm, m, p[2], t192);
    int lz = se_zeroelim(l, t192, p[2], z);
    int lxy = fes_zeroelim(lx, x, ly, y, xy);
    return fes_zeroelim(lxy, xy, lz, z, out);
}

// insphereexact (predicates.hpp:719-984).
float orc_insphere_exact(const float* pa, const float* pb, const float* pc, const float* pd,
                         const float* pe) {
    float ab[4], bc[4], cd[4], de[4], ea[4], ac[4], bd[4], ce[4], da[4], eb[4];
    minor2(pa, pb, ab);
    minor2(pb, pc, bc);
    minor2(pc, pd, cd);
    minor2(pd, pe, de);
    minor2(pe, pa, ea);
    minor2(pa, pc, ac);
    minor2(pb, pd, bd);
    minor2(pc, pe, ce);
    minor2(pd, pa, da);
    minor2(pe, pb, eb);
    float abc[24], bcd[24], cde[24], dea[24], eab[24], abd[24], bce[24], cda[24], deb[24], eac[24];
    int abcl = minor3(bc, pa[2], ac, -pb[2], ab, pc[2], abc);
    int bcdl = minor3(cd, pb[2], bd, -pc[2], bc, pd[2], bcd);
    int cdel = minor3(de, pc[2], ce, -pd[2], cd, pe[2], cde);
    int deal = minor3(ea, pd[2], da, -pe[2], de, pa[2], dea);
    int eabl = minor3(ab, pe[2], eb, -pa[2], ea, pb[2], eab);
    int abdl = minor3(bd, pa[2], da, pb[2], ab, pd[2], abd);
    int bcel = minor3(ce, pb[2], eb, pc[2], bc, pe[2], bce);
    int cdal = minor3(da, pc[2], ac, pd[2], cd, pa[2], cda);
    int debl = minor3(eb, pd[2], bd, pe[2], de, pb[2], deb);
    int eacl = minor3(ac, pe[2], ce, pa[2], ea, pc[2], eac);
    float bcde[96], cdea[96], deab[96], eabc[96], abcd[96];
    int bcdel = minor4(cde, cdel, bce, bcel, deb, debl, bcd, bcdl, bcde);
    int cdeal = minor4(dea, deal, cda, cdal, eac, eacl, cde, cdel, cdea);
    int deabl = minor4(eab, eabl, deb, debl, abd, abdl, dea, deal, deab);
    int eabcl = minor4(abc, abcl, eac, eacl, bce, bcel, eab, eabl, eabc);
    int abcdl = minor4(bcd, bcdl, abd, abdl, cda, cdal, abc, abcl, abcd);
    static __thread float adet[1152], bdet[1152], cdet[1152], ddet[1152], edet[1152];
    static __thread float abdet[2304], cddet[2304], cdedet[3456], det[5760];
    int al = lift(bcde, bcdel, pa, adet);
    int bl = lift(cdea, cdeal, pb, bdet);
    int cl = lift(deab, deabl, pc, cdet);
    int dl = lift(eabc, eabcl, pd, ddet);
    int el = lift(abcd, abcdl, pe, edet);
    int abl = fes_zeroelim(al, adet, bl, bdet, abdet);
    int cdl = fes_zeroelim(cl, cdet, dl, ddet, cddet);
    int cdel2 = fes_zeroelim(cdl, cddet, el, edet, cdedet);
    int n = fes_zeroelim(abl, abdet, cdel2, cdedet, det);
    return det[n - 1];
}

// insphere FP32 filter with its error bound (predicates.hpp:986-1100).
float orc_insphere_filter(const float* pa, const float* pb, const float* pc, const float* pd,
                          const float* pe, float* err) {
    float aex = pa[0] - pe[0], bex = pb[0] - pe[0], cex = pc[0] - pe[0], dex = pd[0] - pe[0];
    float aey = pa[1] - pe[1], bey = pb[1] - pe[1], cey = pc[1] - pe[1], dey = pd[1] - pe[1];
    float aez = pa[2] - pe[2], bez = pb[2] - pe[2], cez = pc[2] - pe[2], dez = pd[2] - pe[2];
    float aexbey = aex * bey, bexaey = bex * aey, ab = aexbey - bexaey;
    float bexcey = bex * cey, cexbey = cex * bey, bc = bexcey - cexbey;
    float cexdey = cex * dey, dexcey = dex * cey, cd = cexdey - dexcey;
    float dexaey = dex * aey, aexdey = aex * dey, da = dexaey - aexdey;
    float aexcey = aex * cey, cexaey = cex * aey, ac = aexcey - cexaey;
    float bexdey = bex * dey, dexbey = dex * bey, bd = bexdey - dexbey;
    float abc = fmaf(aez, bc, fmaf(-bez, ac, cez * ab));
    float bcd = fmaf(bez, cd, fmaf(-cez, bd, dez * bc));
    float cda = fmaf(cez, da, fmaf(dez, ac, aez * cd));
    float dab = fmaf(dez, ab, fmaf(aez, bd, bez * da));
    float alift = fmaf(aex, aex, fmaf(aey, aey, aez * aez));
    float blift = fmaf(bex, bex, fmaf(bey, bey, bez * bez));
    float clift = fmaf(cex, cex, fmaf(cey, cey, cez * cez));
    float dlift = fmaf(dex, dex, fmaf(dey, dey, dez * dez));
    float det = fmaf(dlift, abc, fmaf(-clift, dab, fmaf(blift, cda, (-alift) * bcd)));
    float aezp = fabsf(aez), bezp = fabsf(bez), cezp = fabsf(cez), dezp = fabsf(dez);
    float aexbeyp = fabsf(aexbey), bexaeyp = fabsf(bexaey), bexceyp = fabsf(bexcey);
    float cexbeyp = fabsf(cexbey), cexdeyp = fabsf(cexdey), dexceyp = fabsf(dexcey);
    float dexaeyp = fabsf(dexaey), aexdeyp = fabsf(aexdey), aexceyp = fabsf(aexcey);
    float cexaeyp = fabsf(cexaey), bexdeyp = fabsf(bexdey), dexbeyp = fabsf(dexbey);
    float t_a = fmaf(bezp, (cexdeyp + dexceyp),
                     fmaf(cezp, (dexbeyp + bexdeyp), dezp * (bexceyp + cexbeyp)));
    float t_b = fmaf(cezp, (dexaeyp + aexdeyp),
                     fmaf(dezp, (aexceyp + cexaeyp), aezp * (cexdeyp + dexceyp)));
    float t_c = fmaf(dezp, (aexbeyp + bexaeyp),
                     fmaf(aezp, (bexdeyp + dexbeyp), bezp * (dexaeyp + aexdeyp)));
    float t_d = fmaf(aezp, (bexceyp + cexbeyp),
                     fmaf(bezp, (cexaeyp + aexceyp), cezp * (aexbeyp + bexaeyp)));
    float perm = fmaf(alift, t_a, fmaf(blift, t_b, fmaf(clift, t_c, dlift * t_d)));
    *err = k_isperrboundA * perm;
    return det;
}

// Local Delaunay conflict decision of the star kernel
// (src/mesh/DirectAlphaShape3D.cpp:423-480): the sign of -insphere(a,b,c,d,e)
// with the FP32 filter, then the exact predicate on index-sorted vertices and a
// two-level Simulation of Simplicity on orient3d minors.  ids are the global
// vertex ids used for the ordering; returns the final 'det' of the reference.
float orc_conflict_det(const float* const pts[5], const uint32_t ids[5], int* used_exact) {
    float err;
    float det = -orc_insphere_filter(pts[0], pts[1], pts[2], pts[3], pts[4], &err);
    if (used_exact) *used_exact = 0;
    if (det > err || -det > err) return det;
    if (used_exact) *used_exact = 1;
    uint32_t i[5] = {ids[0], ids[1], ids[2], ids[3], ids[4]};
    const float* p[5] = {pts[0], pts[1], pts[2], pts[3], pts[4]};
    int parity = 0;
    // The 9-exchange sorting network of DirectAlphaShape3D.cpp:447-455.
    static const int net[9][2] = {{0, 4}, {1, 3}, {0, 2}, {2, 4}, {0, 1},
                                  {2, 3}, {1, 4}, {1, 2}, {3, 4}};
    for (int k = 0; k < 9; ++k) {
        int u = net[k][0], v = net[k][1];
        if (i[u] > i[v]) {
            uint32_t t = i[u]; i[u] = i[v]; i[v] = t;
            const float* q = p[u]; p[u] = p[v]; p[v] = q;
            parity ^= 1;
        }
    }
    det = -orc_insphere_exact(p[0], p[1], p[2], p[3], p[4]);
    int depth = 0;
    while (det == 0.0f) {
        ++depth;
        if (depth == 1) det = orc_orient3d(p[1], p[2], p[3], p[4]);
        else if (depth == 2) det = -orc_orient3d(p[0], p[2], p[3], p[4]);
        else det = parity ? 1.0f : -1.0f;
    }
    if (parity) det = -det;
    return det;
}

// ================================ 2D ======================================
// predicates.hpp:337-589.  Bounds as the reference's constexpr initialisers
// compute them (double expressions of the float epsilon, rounded to float).
static const float k_iccerrboundA = (float)((10.0 + 96.0 * (double)ORC_EPS) * (double)ORC_EPS);
static const float k_ccwerrboundA = (float)((3.0 + 16.0 * (double)ORC_EPS) * (double)ORC_EPS);

// (p * q1) - (p * q2) as a 4-component expansion (Two_Product twice, then
// Two_Two_Diff), the 'aterms' / 'bterms' blocks of orient2dexact.
static inline void prod_diff(float p, float q1, float q2, float x[4]) {
    float h1, l1, h2, l2;
    two_product(p, q1, &h1, &l1);
    two_product(p, q2, &h2, &l2);
    two_two_diff(h1, l1, h2, l2, x);
}

// orient2dexact (predicates.hpp:342-383).
float orc_orient2d_exact(const float* pa, const float* pb, const float* pc) {
    float at[4], bt[4], v[8], w[12];
    prod_diff(pa[0], pb[1], pc[1], at);  // ax*by - ax*cy
    prod_diff(pb[0], pc[1], pa[1], bt);  // bx*cy - bx*ay
    const int vl = fes_zeroelim(4, at, 4, bt, v);
    prod_diff(pc[0], pa[1], pb[1], at);  // cx*ay - cx*by
    const int wl = fes_zeroelim(vl, v, 4, at, w);
    return w[wl - 1];
}

// orient2d with its stage-A filter (predicates.hpp:385-418).
float orc_orient2d(const float* pa, const float* pb, const float* pc) {
    const float detleft = (pa[0] - pc[0]) * (pb[1] - pc[1]);
    const float detright = (pa[1] - pc[1]) * (pb[0] - pc[0]);
    const float det = detleft - detright;
    float detsum;
    if (detleft > 0.0f) {
        if (detright <= 0.0f) return det;
        detsum = detleft + detright;
    } else if (detleft < 0.0f) {
        if (detright >= 0.0f) return det;
        detsum = -detleft - detright;
    } else {
        return det;
    }
    const float errbound = k_ccwerrboundA * detsum;
    if ((det >= errbound) || (-det >= errbound)) return det;
    return orc_orient2d_exact(pa, pb, pc);
}

// incircle FP32 filter (predicates.hpp:544-586), explicit fmaf as written there.
float orc_incircle_filter(const float* pa, const float* pb, const float* pc, const float* pd, float* err) {
    const float adx = pa[0] - pd[0], bdx = pb[0] - pd[0], cdx = pc[0] - pd[0];
    const float ady = pa[1] - pd[1], bdy = pb[1] - pd[1], cdy = pc[1] - pd[1];
    const float bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    const float alift = fmaf(adx, adx, ady * ady);
    const float cdxady = cdx * ady, adxcdy = adx * cdy;
    const float blift = fmaf(bdx, bdx, bdy * bdy);
    const float adxbdy = adx * bdy, bdxady = bdx * ady;
    const float clift = fmaf(cdx, cdx, cdy * cdy);
    const float det = fmaf(alift, (bdxcdy - cdxbdy), fmaf(blift, (cdxady - adxcdy), clift * (adxbdy - bdxady)));
    const float permanent = fmaf(alift, (fabsf(bdxcdy) + fabsf(cdxbdy)),
                                 fmaf(blift, (fabsf(cdxady) + fabsf(adxcdy)), (fabsf(adxbdy) + fabsf(bdxady)) * clift));
    *err = k_iccerrboundA * permanent;
    return det;
}

// lift * m as the reference forms it: (m * x) * (sx x) + (m * y) * (sy y), sx, sy = +-1.
static int lift2(const float* m, int lm, const float* p, float sign, float* out) {
    float d24x[24], d24y[24], d48x[48], d48y[48];
    int xl = se_zeroelim(lm, m, p[0], d24x);
    xl = se_zeroelim(xl, d24x, sign * p[0], d48x);
    int yl = se_zeroelim(lm, m, p[1], d24y);
    yl = se_zeroelim(yl, d24y, sign * p[1], d48y);
    return fes_zeroelim(xl, d48x, yl, d48y, out);
}

// incircleexact (predicates.hpp:420-542), same expansion sequence.
float orc_incircle_exact(const float* pa, const float* pb, const float* pc, const float* pd) {
    float ab[4], bc[4], cd[4], da[4], ac[4], bd[4];
    minor2(pa, pb, ab);
    minor2(pb, pc, bc);
    minor2(pc, pd, cd);
    minor2(pd, pa, da);
    minor2(pa, pc, ac);
    minor2(pb, pd, bd);
    float t8[8], abc[12], bcd[12], cda[12], dab[12];
    int tl = fes_zeroelim(4, cd, 4, da, t8);
    const int cdal = fes_zeroelim(tl, t8, 4, ac, cda);
    tl = fes_zeroelim(4, da, 4, ab, t8);
    const int dabl = fes_zeroelim(tl, t8, 4, bd, dab);
    for (int i = 0; i < 4; ++i) {
        bd[i] = -bd[i];
        ac[i] = -ac[i];
    }
    tl = fes_zeroelim(4, ab, 4, bc, t8);
    const int abcl = fes_zeroelim(tl, t8, 4, ac, abc);
    tl = fes_zeroelim(4, bc, 4, cd, t8);
    const int bcdl = fes_zeroelim(tl, t8, 4, bd, bcd);
    float adet[96], bdet[96], abdet[192], cddet[192], deter[384];
    const int al = lift2(bcd, bcdl, pa, 1.0f, adet);
    const int bl = lift2(cda, cdal, pb, -1.0f, bdet);
    const int abl = fes_zeroelim(al, adet, bl, bdet, abdet);
    const int cl = lift2(dab, dabl, pc, 1.0f, adet);
    const int dl = lift2(abc, abcl, pd, -1.0f, bdet);
    const int cdl = fes_zeroelim(cl, adet, dl, bdet, cddet);
    const int n = fes_zeroelim(abl, abdet, cdl, cddet, deter);
    return deter[n - 1];
}
