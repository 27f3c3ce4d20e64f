// Geometric predicates of the star Delaunay kernel (device side).
//
// Decision procedure for "is point e inside the circumsphere of (a,b,c,d)"
// as the reference's star kernel takes it (src/mesh/DirectAlphaShape3D.cpp:
// 423-480, predicates from include/geometry/predicates.hpp):
//   1. FP32 filter with its error bound (predicates.hpp:986-1100): identical
//      float operations, so its "certain" answers are the reference's.
//   2. FP64 semi-static filter (new).  Used only when every coordinate of the
//      five points is 0 or has magnitude in [2^-6, 2^20): then every product
//      of five coordinates is a multiple of 2^-145, so the reference's FP32
//      expansions cannot underflow and its "exact" answer is the true sign,
//      which a certain FP64 filter also gives.  Coordinate differences are
//      exact in FP64 for that range.
//   3. FP32 exact expansions (Shewchuk's published algorithm as restated by
//      predicates.hpp:229-335,591-984) on index-sorted vertices, then the
//      reference's two-level Simulation of Simplicity on orient3d minors.
// Stage 3 repeats the reference's float operation sequence exactly so that
// its answers (including any FP32 tail underflow near the origin) match.
//
// All functions assume compilation with -fmad=false; explicit fmaf() calls
// stay fused as in the reference.
#pragma once

#include <cstdint>

#include "common.cuh"

#include "exact_int.cuh"

namespace sb {
namespace pred {

constexpr float kSplitter = 4097.0f;
constexpr float kEps = 5.9604644775390625e-08f;
// predicates.hpp:588-589: double expressions of the float epsilon, rounded to float.
constexpr float kIspErrA = (float)((16.0 + 224.0 * (double)kEps) * (double)kEps);
constexpr float kO3dErrA = (float)((7.0 + 56.0 * (double)kEps) * (double)kEps);

// ------------------------------------------------------- FP32 filters ----
// The determinant of the FP32 insphere filter (predicates.hpp:986-1100).
__device__ __forceinline__ float insphere32_det(const float3 a, const float3 b, const float3 c, const float3 d,
                                                const float3 e) {
    const float aex = a.x - e.x, bex = b.x - e.x, cex = c.x - e.x, dex = d.x - e.x;
    const float aey = a.y - e.y, bey = b.y - e.y, cey = c.y - e.y, dey = d.y - e.y;
    const float aez = a.z - e.z, bez = b.z - e.z, cez = c.z - e.z, dez = d.z - e.z;
    const float ab = aex * bey - bex * aey, bc = bex * cey - cex * bey, cd = cex * dey - dex * cey;
    const float da = dex * aey - aex * dey, ac = aex * cey - cex * aey, bd = bex * dey - dex * bey;
    const float abc = fmaf(aez, bc, fmaf(-bez, ac, cez * ab));
    const float bcd = fmaf(bez, cd, fmaf(-cez, bd, dez * bc));
    const float cda = fmaf(cez, da, fmaf(dez, ac, aez * cd));
    const float dab = fmaf(dez, ab, fmaf(aez, bd, bez * da));
    const float alift = fmaf(aex, aex, fmaf(aey, aey, aez * aez));
    const float blift = fmaf(bex, bex, fmaf(bey, bey, bez * bez));
    const float clift = fmaf(cex, cex, fmaf(cey, cey, cez * cez));
    const float dlift = fmaf(dex, dex, fmaf(dey, dey, dez * dez));
    return fmaf(dlift, abc, fmaf(-clift, dab, fmaf(blift, cda, (-alift) * bcd)));
}

// The filter: its determinant and its error bound err = kIspErrA x permanent.
__device__ __forceinline__ float insphere32(const float3 a, const float3 b, const float3 c, const float3 d,
                                            const float3 e, float& err) {
    const float det = insphere32_det(a, b, c, d, e);
    const float aex = a.x - e.x, bex = b.x - e.x, cex = c.x - e.x, dex = d.x - e.x;
    const float aey = a.y - e.y, bey = b.y - e.y, cey = c.y - e.y, dey = d.y - e.y;
    const float aez = a.z - e.z, bez = b.z - e.z, cez = c.z - e.z, dez = d.z - e.z;
    const float aexbey = aex * bey, bexaey = bex * aey, bexcey = bex * cey, cexbey = cex * bey;
    const float cexdey = cex * dey, dexcey = dex * cey, dexaey = dex * aey, aexdey = aex * dey;
    const float aexcey = aex * cey, cexaey = cex * aey, bexdey = bex * dey, dexbey = dex * bey;
    const float alift = fmaf(aex, aex, fmaf(aey, aey, aez * aez));
    const float blift = fmaf(bex, bex, fmaf(bey, bey, bez * bez));
    const float clift = fmaf(cex, cex, fmaf(cey, cey, cez * cez));
    const float dlift = fmaf(dex, dex, fmaf(dey, dey, dez * dez));
    const float aezp = fabsf(aez), bezp = fabsf(bez), cezp = fabsf(cez), dezp = fabsf(dez);
    const float aexbeyp = fabsf(aexbey), bexaeyp = fabsf(bexaey), bexceyp = fabsf(bexcey);
    const float cexbeyp = fabsf(cexbey), cexdeyp = fabsf(cexdey), dexceyp = fabsf(dexcey);
    const float dexaeyp = fabsf(dexaey), aexdeyp = fabsf(aexdey), aexceyp = fabsf(aexcey);
    const float cexaeyp = fabsf(cexaey), bexdeyp = fabsf(bexdey), dexbeyp = fabsf(dexbey);
    const float ta = fmaf(bezp, (cexdeyp + dexceyp), fmaf(cezp, (dexbeyp + bexdeyp), dezp * (bexceyp + cexbeyp)));
    const float tb = fmaf(cezp, (dexaeyp + aexdeyp), fmaf(dezp, (aexceyp + cexaeyp), aezp * (cexdeyp + dexceyp)));
    const float tc = fmaf(dezp, (aexbeyp + bexaeyp), fmaf(aezp, (bexdeyp + dexbeyp), bezp * (dexaeyp + aexdeyp)));
    const float td = fmaf(aezp, (bexceyp + cexbeyp), fmaf(bezp, (cexaeyp + aexceyp), cezp * (aexbeyp + bexaeyp)));
    const float perm = fmaf(alift, ta, fmaf(blift, tb, fmaf(clift, tc, dlift * td)));
    err = kIspErrA * perm;
    return det;
}

// An upper bound of the filter's err for every test of one star whose finite
// points all lie within mc of the star centre in each coordinate, so that a
// test can skip the permanent: |det| above the bound is above err, and the
// filter is certain with the same det.  Every coordinate difference the filter
// forms is then at most 2 mc before rounding and D = 2 mc (1 + 2^-20) after
// (mc itself is a rounded maximum); each lift is at most 3 D^2 and each
// bracketed sum of the permanent (ta ... td) at most 6 D^3, so the permanent
// is at most 72 D^5, and its ten roundings and the one of kIspErrA x perm add
// less than the factor 1 + 2^-16.  Products that underflow lose at most
// 2^-150 each, which the added 2^-120 covers.  Outside mc in [2^-21, 2^19)
// the bound is INFINITY (no test skips the permanent).
__device__ __forceinline__ float star_filter_bound(float mc) {
    if (!(mc >= 0x1p-21f && mc < 0x1p19f)) return INFINITY;
    const double D = 2.0 * (double)mc * (1.0 + 0x1p-20), D2 = D * D;
    return __double2float_ru((double)kIspErrA * 72.0 * (D2 * D2 * D) * (1.0 + 0x1p-16) + 0x1p-120);
}

// ------------------------------------------------------- FP64 filter -----
// Stage 2 may only decide where the reference's stage 3 (FP32 expansion
// arithmetic) returns the true sign.  Those expansions are exact unless a
// product underflows, which loses at most 2^-150 per product, far below
// 2^-120 in all; and they do not overflow while every coordinate is below
// 2^20.  So stage 2 applies when every coordinate is 0 or in [2^-60, 2^20)
// (every degree-5 term then stays in double's normal range), and it decides
// only when |det| exceeds its error bound plus 2^-120.  Its differences are
// rounded (relative error <= eps, exact when the operands are close), which
// moves each degree-5 term by at most 5 eps of its magnitude: the bound is
// Shewchuk's isperrboundA ((16 + 224 eps) eps x permanent) with 32 + 512 eps
// instead.  Where every coordinate is 0 or at least 2^-6 the reference's
// expansions cannot underflow at all (all their terms are multiples of
// 2^-145); that narrower range sent every test near a face of the unit cube
// to the exact stage (729 undecided stars of the 1M dam-break column, 2.7 ms
// of exact pass at 4M).
constexpr double kIspErrA64Wide = (32.0 + 512.0 * 1.1102230246251565e-16) * 1.1102230246251565e-16;
constexpr double kStage3Loss = 0x1p-120;
__device__ __forceinline__ bool safe_coord(float x) {
    const float ax = fabsf(x);
    return x == 0.0f || (ax >= 0x1p-60f && ax < 1048576.0f);
}
__device__ __forceinline__ bool fp64_applicable(const float3 a, const float3 b, const float3 c, const float3 d,
                                                const float3 e) {
    return safe_coord(a.x) && safe_coord(a.y) && safe_coord(a.z) && safe_coord(b.x) && safe_coord(b.y) &&
           safe_coord(b.z) && safe_coord(c.x) && safe_coord(c.y) && safe_coord(c.z) && safe_coord(d.x) &&
           safe_coord(d.y) && safe_coord(d.z) && safe_coord(e.x) && safe_coord(e.y) && safe_coord(e.z);
}
// Shewchuk's insphere stage-A expression in double (no contraction) with the
// bound above.  Returns +1/-1 when the sign of insphere(a,b,c,d,e) is
// certain, 0 otherwise.
__device__ __forceinline__ int insphere64_sign(const float3 a, const float3 b, const float3 c, const float3 d,
                                               const float3 e) {
    const double aex = (double)a.x - e.x, bex = (double)b.x - e.x, cex = (double)c.x - e.x, dex = (double)d.x - e.x;
    const double aey = (double)a.y - e.y, bey = (double)b.y - e.y, cey = (double)c.y - e.y, dey = (double)d.y - e.y;
    const double aez = (double)a.z - e.z, bez = (double)b.z - e.z, cez = (double)c.z - e.z, dez = (double)d.z - e.z;
    const double aexbey = aex * bey, bexaey = bex * aey, ab = aexbey - bexaey;
    const double bexcey = bex * cey, cexbey = cex * bey, bc = bexcey - cexbey;
    const double cexdey = cex * dey, dexcey = dex * cey, cd = cexdey - dexcey;
    const double dexaey = dex * aey, aexdey = aex * dey, da = dexaey - aexdey;
    const double aexcey = aex * cey, cexaey = cex * aey, ac = aexcey - cexaey;
    const double bexdey = bex * dey, dexbey = dex * bey, bd = bexdey - dexbey;
    const double abc = aez * bc - bez * ac + cez * ab;
    const double bcd = bez * cd - cez * bd + dez * bc;
    const double cda = cez * da + dez * ac + aez * cd;
    const double dab = dez * ab + aez * bd + bez * da;
    const double alift = aex * aex + aey * aey + aez * aez;
    const double blift = bex * bex + bey * bey + bez * bez;
    const double clift = cex * cex + cey * cey + cez * cez;
    const double dlift = dex * dex + dey * dey + dez * dez;
    const double det = (dlift * abc - clift * dab) + (blift * cda - alift * bcd);
    const double aezp = fabs(aez), bezp = fabs(bez), cezp = fabs(cez), dezp = fabs(dez);
    const double aexbeyp = fabs(aexbey), bexaeyp = fabs(bexaey), bexceyp = fabs(bexcey);
    const double cexbeyp = fabs(cexbey), cexdeyp = fabs(cexdey), dexceyp = fabs(dexcey);
    const double dexaeyp = fabs(dexaey), aexdeyp = fabs(aexdey), aexceyp = fabs(aexcey);
    const double cexaeyp = fabs(cexaey), bexdeyp = fabs(bexdey), dexbeyp = fabs(dexbey);
    const double perm = ((cexdeyp + dexceyp) * bezp + (dexbeyp + bexdeyp) * cezp + (bexceyp + cexbeyp) * dezp) * alift +
                        ((dexaeyp + aexdeyp) * cezp + (aexceyp + cexaeyp) * dezp + (cexdeyp + dexceyp) * aezp) * blift +
                        ((aexbeyp + bexaeyp) * dezp + (bexdeyp + dexbeyp) * aezp + (dexaeyp + aexdeyp) * bezp) * clift +
                        ((bexceyp + cexbeyp) * aezp + (cexaeyp + aexceyp) * bezp + (aexbeyp + bexaeyp) * cezp) * dlift;
    const double eb = kIspErrA64Wide * perm + kStage3Loss;
    if (det > eb) return 1;
    if (-det > eb) return -1;
    return 0;
}

// -------------------------------------------- FP32 exact expansions -------
// Error-free transformations with the operation order of the reference's
// macros (predicates.hpp:29-88).
__device__ __forceinline__ void two_sum(float a, float b, float& x, float& y) {
    x = a + b;
    const float bv = x - a, av = x - bv, br = b - bv, ar = a - av;
    y = ar + br;
}
__device__ __forceinline__ void fast_two_sum(float a, float b, float& x, float& y) {
    x = a + b;
    const float bv = x - a;
    y = b - bv;
}
__device__ __forceinline__ void two_diff(float a, float b, float& x, float& y) {
    x = a - b;
    const float bv = a - x, av = x + bv, br = bv - b, ar = a - av;
    y = ar + br;
}
__device__ __forceinline__ void split(float a, float& hi, float& lo) {
    const float c = kSplitter * a, big = c - a;
    hi = c - big;
    lo = a - hi;
}
__device__ __forceinline__ void two_product_presplit(float a, float b, float bhi, float blo, float& x, float& y) {
    x = a * b;
    float ahi, alo;
    split(a, ahi, alo);
    const float e1 = x - (ahi * bhi), e2 = e1 - (alo * bhi), e3 = e2 - (ahi * blo);
    y = (alo * blo) - e3;
}
__device__ __forceinline__ void two_product(float a, float b, float& x, float& y) {
    float bhi, blo;
    split(b, bhi, blo);
    two_product_presplit(a, b, bhi, blo, x, y);
}
// p.x*q.y - q.x*p.y as a 4-term expansion (Two_Product + Two_Two_Diff).
__device__ __forceinline__ void minor2(const float3 p, const float3 q, float m[4]) {
    float h1, l1, h2, l2, i, j, z;
    two_product(p.x, q.y, h1, l1);
    two_product(q.x, p.y, h2, l2);
    two_diff(l1, l2, i, m[0]);
    two_sum(h1, i, j, z);
    two_diff(z, h2, i, m[1]);
    two_sum(j, i, m[3], m[2]);
}

// Capacity of the long expansion buffers of insphere_exact and the scratch it
// needs (floats) per call.
constexpr int kExpCap = 288;
constexpr int kInsphereScratchFloats = 40 + 240 + 480 + 96 + 32 + 192 + 4 * kExpCap + 4 * kExpCap;

// Expansion sum with zero elimination (fast_expansion_sum_zeroelim,
// predicates.hpp:229-296).  h holds at most `cap` terms; a longer result sets
// ST_EXACT_OVERFLOW (never expected: a nonoverlapping float expansion has at
// most 277 nonzero terms).
static __device__ __noinline__ int fes(int elen, const float* e, int flen, const float* f, float* h, int cap,
                                uint32_t& st) {
    float Q, Qn, hh;
    int ei = 0, fi = 0, hi = 0;
    float en = e[0], fn = f[0];
#define SB_NEXT_E() (en = (++ei < elen) ? e[ei] : 0.0f)
#define SB_NEXT_F() (fn = (++fi < flen) ? f[fi] : 0.0f)
#define SB_PUT(v) do { if (hi < cap) h[hi] = (v); else st |= ST_EXACT_OVERFLOW; ++hi; } while (0)
    if ((fn > en) == (fn > -en)) { Q = en; SB_NEXT_E(); }
    else { Q = fn; SB_NEXT_F(); }
    if (ei < elen && fi < flen) {
        if ((fn > en) == (fn > -en)) { fast_two_sum(en, Q, Qn, hh); SB_NEXT_E(); }
        else { fast_two_sum(fn, Q, Qn, hh); SB_NEXT_F(); }
        Q = Qn;
        if (hh != 0.0f) SB_PUT(hh);
        while (ei < elen && fi < flen) {
            if ((fn > en) == (fn > -en)) { two_sum(Q, en, Qn, hh); SB_NEXT_E(); }
            else { two_sum(Q, fn, Qn, hh); SB_NEXT_F(); }
            Q = Qn;
            if (hh != 0.0f) SB_PUT(hh);
        }
    }
    while (ei < elen) {
        two_sum(Q, en, Qn, hh);
        SB_NEXT_E();
        Q = Qn;
        if (hh != 0.0f) SB_PUT(hh);
    }
    while (fi < flen) {
        two_sum(Q, fn, Qn, hh);
        SB_NEXT_F();
        Q = Qn;
        if (hh != 0.0f) SB_PUT(hh);
    }
    if (Q != 0.0f || hi == 0) SB_PUT(Q);
    return hi < cap ? hi : cap;
}

// scale_expansion_zeroelim (predicates.hpp:298-335).
static __device__ __noinline__ int sez(int elen, const float* e, float b, float* h, int cap, uint32_t& st) {
    float bhi, blo, Q, hh, p1, p0, s;
    split(b, bhi, blo);
    two_product_presplit(e[0], b, bhi, blo, Q, hh);
    int hi = 0;
    if (hh != 0.0f) SB_PUT(hh);
    for (int i = 1; i < elen; ++i) {
        two_product_presplit(e[i], b, bhi, blo, p1, p0);
        two_sum(Q, p0, s, hh);
        if (hh != 0.0f) SB_PUT(hh);
        fast_two_sum(p1, s, Q, hh);
        if (hh != 0.0f) SB_PUT(hh);
    }
    if (Q != 0.0f || hi == 0) SB_PUT(Q);
    return hi < cap ? hi : cap;
#undef SB_NEXT_E
#undef SB_NEXT_F
#undef SB_PUT
}

// orient3dexact (predicates.hpp:591-670).
static __device__ __noinline__ float orient3d_exact(const float3 a, const float3 b, const float3 c, const float3 d,
                                             uint32_t& st) {
    float ab[4], bc[4], cd[4], da[4], ac[4], bd[4];
    float t8[8], abc[12], bcd[12], cda[12], dab[12];
    float adet[24], bdet[24], cdet[24], ddet[24], abdet[48], cddet[48], det[96];
    minor2(a, b, ab);
    minor2(b, c, bc);
    minor2(c, d, cd);
    minor2(d, a, da);
    minor2(a, c, ac);
    minor2(b, d, bd);
    int tl = fes(4, cd, 4, da, t8, 8, st);
    const int cdal = fes(tl, t8, 4, ac, cda, 12, st);
    tl = fes(4, da, 4, ab, t8, 8, st);
    const int dabl = fes(tl, t8, 4, bd, dab, 12, st);
    for (int i = 0; i < 4; ++i) { bd[i] = -bd[i]; ac[i] = -ac[i]; }
    tl = fes(4, ab, 4, bc, t8, 8, st);
    const int abcl = fes(tl, t8, 4, ac, abc, 12, st);
    tl = fes(4, bc, 4, cd, t8, 8, st);
    const int bcdl = fes(tl, t8, 4, bd, bcd, 12, st);
    const int al = sez(bcdl, bcd, a.z, adet, 24, st);
    const int bl = sez(cdal, cda, -b.z, bdet, 24, st);
    const int cl = sez(dabl, dab, c.z, cdet, 24, st);
    const int dl = sez(abcl, abc, -d.z, ddet, 24, st);
    const int abl = fes(al, adet, bl, bdet, abdet, 48, st);
    const int cdl = fes(cl, cdet, dl, ddet, cddet, 48, st);
    const int n = fes(abl, abdet, cdl, cddet, det, 96, st);
    return det[n - 1];
}

// orient3d: FP32 filter then exact (predicates.hpp:671-714).
__device__ __forceinline__ float orient3d(const float3 a, const float3 b, const float3 c, const float3 d,
                                          uint32_t& st) {
    const float adx = a.x - d.x, bdx = b.x - d.x, cdx = c.x - d.x;
    const float ady = a.y - d.y, bdy = b.y - d.y, cdy = c.y - d.y;
    const float adz = a.z - d.z, bdz = b.z - d.z, cdz = c.z - d.z;
    const float bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    const float cdxady = cdx * ady, adxcdy = adx * cdy;
    const float adxbdy = adx * bdy, bdxady = bdx * ady;
    const float det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
    const float perm = (fabsf(bdxcdy) + fabsf(cdxbdy)) * fabsf(adz) + (fabsf(cdxady) + fabsf(adxcdy)) * fabsf(bdz) +
                       (fabsf(adxbdy) + fabsf(bdxady)) * fabsf(cdz);
    const float eb = kO3dErrA * perm;
    if (det > eb || -det > eb) return det;
    if (xint::coord_ok(a.x) && xint::coord_ok(a.y) && xint::coord_ok(a.z) && xint::coord_ok(b.x) &&
        xint::coord_ok(b.y) && xint::coord_ok(b.z) && xint::coord_ok(c.x) && xint::coord_ok(c.y) &&
        xint::coord_ok(c.z) && xint::coord_ok(d.x) && xint::coord_ok(d.y) && xint::coord_ok(d.z))
        return (float)xint::orient3d_sign(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z, d.x, d.y, d.z);
    return orient3d_exact(a, b, c, d, st);
}

// 3x3 minor s3*M3 + (s1*M1 + s2*M2) (predicates.hpp:818-876).
__device__ __forceinline__ int minor3(const float* m1, float s1, const float* m2, float s2, const float* m3, float s3,
                                      float* out, float* t8a, float* t8b, float* t16, uint32_t& st) {
    int la = sez(4, m1, s1, t8a, 8, st);
    const int lb = sez(4, m2, s2, t8b, 8, st);
    const int l16 = fes(la, t8a, lb, t8b, t16, 16, st);
    la = sez(4, m3, s3, t8a, 8, st);
    return fes(la, t8a, l16, t16, out, 24, st);
}
// (p + q) - (r + s) (predicates.hpp:878-956).
__device__ __forceinline__ int minor4(const float* p, int lp, const float* q, int lq, const float* r, int lr,
                                      const float* s, int ls, float* out, float* a, float* b, uint32_t& st) {
    const int la = fes(lp, p, lq, q, a, 48, st);
    const int lb = fes(lr, r, ls, s, b, 48, st);
    for (int i = 0; i < lb; ++i) b[i] = -b[i];
    return fes(la, a, lb, b, out, 96, st);
}
// m * (px^2 + py^2 + pz^2): x, y, z partial products, then (x + y) + z.
__device__ __forceinline__ int lift(const float* m, int lm, const float3 p, float* out, float* t192, float* x,
                                    float* y, float* z, float* xy, uint32_t& st) {
    int l = sez(lm, m, p.x, t192, 192, st);
    const int lx = sez(l, t192, p.x, x, kExpCap, st);
    l = sez(lm, m, p.y, t192, 192, st);
    const int ly = sez(l, t192, p.y, y, kExpCap, st);
    l = sez(lm, m, p.z, t192, 192, st);
    const int lz = sez(l, t192, p.z, z, kExpCap, st);
    const int lxy = fes(lx, x, ly, y, xy, kExpCap, st);
    return fes(lxy, xy, lz, z, out, kExpCap, st);
}

// insphereexact (predicates.hpp:719-984) on caller-provided scratch.
static __device__ __noinline__ float insphere_exact(const float3 a, const float3 b, const float3 c, const float3 d,
                                             const float3 e, float* w, uint32_t& st) {
    float* m2 = w;            // 10 x 4
    float* m3 = m2 + 40;      // 10 x 24
    float* m4 = m3 + 240;     // 5 x 96
    float* t48a = m4 + 480;   // 48
    float* t48b = t48a + 48;  // 48
    float* t8a = t48b + 48;   // 8
    float* t8b = t8a + 8;     // 8
    float* t16 = t8b + 8;     // 16
    float* t192 = t16 + 16;   // 192
    float* x = t192 + 192;
    float* y = x + kExpCap;
    float* z = y + kExpCap;
    float* xy = z + kExpCap;
    float* P = xy + kExpCap;
    float* Q = P + kExpCap;
    float* R = Q + kExpCap;
    float* AB = R + kExpCap;
    float *ab = m2, *bc = m2 + 4, *cd = m2 + 8, *de = m2 + 12, *ea = m2 + 16;
    float *ac = m2 + 20, *bd = m2 + 24, *ce = m2 + 28, *da = m2 + 32, *eb = m2 + 36;
    minor2(a, b, ab);
    minor2(b, c, bc);
    minor2(c, d, cd);
    minor2(d, e, de);
    minor2(e, a, ea);
    minor2(a, c, ac);
    minor2(b, d, bd);
    minor2(c, e, ce);
    minor2(d, a, da);
    minor2(e, b, eb);
    float *abc = m3, *bcd = m3 + 24, *cde = m3 + 48, *dea = m3 + 72, *eab = m3 + 96;
    float *abd = m3 + 120, *bce = m3 + 144, *cda = m3 + 168, *deb = m3 + 192, *eac = m3 + 216;
    const int abcl = minor3(bc, a.z, ac, -b.z, ab, c.z, abc, t8a, t8b, t16, st);
    const int bcdl = minor3(cd, b.z, bd, -c.z, bc, d.z, bcd, t8a, t8b, t16, st);
    const int cdel = minor3(de, c.z, ce, -d.z, cd, e.z, cde, t8a, t8b, t16, st);
    const int deal = minor3(ea, d.z, da, -e.z, de, a.z, dea, t8a, t8b, t16, st);
    const int eabl = minor3(ab, e.z, eb, -a.z, ea, b.z, eab, t8a, t8b, t16, st);
    const int abdl = minor3(bd, a.z, da, b.z, ab, d.z, abd, t8a, t8b, t16, st);
    const int bcel = minor3(ce, b.z, eb, c.z, bc, e.z, bce, t8a, t8b, t16, st);
    const int cdal = minor3(da, c.z, ac, d.z, cd, a.z, cda, t8a, t8b, t16, st);
    const int debl = minor3(eb, d.z, bd, e.z, de, b.z, deb, t8a, t8b, t16, st);
    const int eacl = minor3(ac, e.z, ce, a.z, ea, c.z, eac, t8a, t8b, t16, st);
    float *bcde = m4, *cdea = m4 + 96, *deab = m4 + 192, *eabc = m4 + 288, *abcd = m4 + 384;
    const int bcdel = minor4(cde, cdel, bce, bcel, deb, debl, bcd, bcdl, bcde, t48a, t48b, st);
    const int cdeal = minor4(dea, deal, cda, cdal, eac, eacl, cde, cdel, cdea, t48a, t48b, st);
    const int deabl = minor4(eab, eabl, deb, debl, abd, abdl, dea, deal, deab, t48a, t48b, st);
    const int eabcl = minor4(abc, abcl, eac, eacl, bce, bcel, eab, eabl, eabc, t48a, t48b, st);
    const int abcdl = minor4(bcd, bcdl, abd, abdl, cda, cdal, abc, abcl, abcd, t48a, t48b, st);
    // adet + bdet -> AB; cdet + ddet -> R; R + edet -> Q; AB + Q -> P.
    const int al = lift(bcde, bcdel, a, P, t192, x, y, z, xy, st);
    const int bl = lift(cdea, cdeal, b, Q, t192, x, y, z, xy, st);
    const int abl = fes(al, P, bl, Q, AB, kExpCap, st);
    const int cl = lift(deab, deabl, c, P, t192, x, y, z, xy, st);
    const int dl = lift(eabc, eabcl, d, Q, t192, x, y, z, xy, st);
    const int cdl = fes(cl, P, dl, Q, R, kExpCap, st);
    const int el = lift(abcd, abcdl, e, P, t192, x, y, z, xy, st);
    const int cdel2 = fes(cdl, R, el, P, Q, kExpCap, st);
    const int n = fes(abl, AB, cdel2, Q, P, kExpCap, st);
    return P[n - 1];
}

// Stage 3 (exact expansions + SoS) on caller-provided scratch.
static __device__ __noinline__ float conflict_exact(const float3 (&pin)[5], const uint32_t (&idin)[5], float* scratch,
                                                    uint32_t& st) {
    uint32_t i[5] = {idin[0], idin[1], idin[2], idin[3], idin[4]};
    float3 q[5] = {pin[0], pin[1], pin[2], pin[3], pin[4]};
    bool swp = false;
    // 9-exchange sorting network of DirectAlphaShape3D.cpp:447-455.
#define SB_CX(u, v) if (i[u] > i[v]) { uint32_t t_ = i[u]; i[u] = i[v]; i[v] = t_; float3 f_ = q[u]; q[u] = q[v]; q[v] = f_; swp = !swp; }
    SB_CX(0, 4) SB_CX(1, 3) SB_CX(0, 2) SB_CX(2, 4) SB_CX(0, 1) SB_CX(2, 3) SB_CX(1, 4) SB_CX(1, 2) SB_CX(3, 4)
#undef SB_CX
    bool in_range = true;
#pragma unroll
    for (int k = 0; k < 5; ++k)
        in_range = in_range && xint::coord_ok(q[k].x) && xint::coord_ok(q[k].y) && xint::coord_ok(q[k].z);
    float det;
    if (in_range) {  // the reference's expansions are exact there: the fixed-point sign is theirs
        const float qa[3] = {q[0].x, q[0].y, q[0].z}, qb[3] = {q[1].x, q[1].y, q[1].z};
        const float qc[3] = {q[2].x, q[2].y, q[2].z}, qd[3] = {q[3].x, q[3].y, q[3].z};
        const float qe[3] = {q[4].x, q[4].y, q[4].z};
        det = -(float)xint::insphere_sign(qa, qb, qc, qd, qe);
    } else {
        det = -insphere_exact(q[0], q[1], q[2], q[3], q[4], scratch, st);
    }
    int depth = 0;
    while (det == 0.0f) {
        ++depth;
        if (depth == 1) det = orient3d(q[1], q[2], q[3], q[4], st);
        else if (depth == 2) det = -orient3d(q[0], q[2], q[3], q[4], st);
        else det = swp ? 1.0f : -1.0f;
    }
    if (swp) det = -det;
    return det;
}

// Stage 3 with its scratch in this call's own stack frame (per-thread local
// memory), for kernels that evaluate the exact stage in place.
static __device__ __noinline__ float conflict_exact_local(const float3 (&pin)[5], const uint32_t (&idin)[5],
                                                          uint32_t& st) {
    float w[kInsphereScratchFloats];
    return conflict_exact(pin, idin, w, st);
}

// Stages 1-2.  Returns true and sets det when decided.
__device__ __forceinline__ bool conflict_fast(const float3 p[5], float& det) {
    float err;
    const float det32 = -insphere32(p[0], p[1], p[2], p[3], p[4], err);
    if (det32 > err || -det32 > err) { det = det32; return true; }
    if (fp64_applicable(p[0], p[1], p[2], p[3], p[4])) {
        const int s = insphere64_sign(p[0], p[1], p[2], p[3], p[4]);
        if (s != 0) { det = s > 0 ? -1.0f : 1.0f; return true; }  // det = -insphere
    }
    return false;
}

// Stages 1-2 as conflict_fast, also counting the FP64 filter evaluations (the
// work counters of profiling runs).
__device__ __forceinline__ bool conflict_fast_count(const float3 p[5], float& det, uint32_t& n64) {
    float err;
    const float det32 = -insphere32(p[0], p[1], p[2], p[3], p[4], err);
    if (det32 > err || -det32 > err) { det = det32; return true; }
    if (fp64_applicable(p[0], p[1], p[2], p[3], p[4])) {
        ++n64;
        const int s = insphere64_sign(p[0], p[1], p[2], p[3], p[4]);
        if (s != 0) { det = s > 0 ? -1.0f : 1.0f; return true; }
    }
    return false;
}
// Floating-point operations of one insphere32 (FMA = 2): 12 coordinate
// differences, 6 minors (18), 4 3x3 minors (20), 4 lifts (20), det (7), the
// permanent and its bound (40).  insphere64_sign performs the same count in FP64.
constexpr uint32_t kInsphereFlops = 117;

// Reference decision (DirectAlphaShape3D.cpp:423-480) for vertices p[0..4]
// with global ids ids[0..4] (p[0] the star centre, p[4] the inserted point).
// Returns the reference's 'det' (only its sign is meaningful).  The exact
// stage uses `scratch` (kInsphereScratchFloats floats) if given, else its own
// stack frame.
__device__ __forceinline__ float conflict_det(const float3 (&p)[5], const uint32_t (&ids)[5], float* scratch,
                                              bool& need_exact, uint32_t& st, uint32_t& n_exact) {
    need_exact = false;
    float det;
    if (conflict_fast(p, det)) return det;
    ++n_exact;
    return scratch ? conflict_exact(p, ids, scratch, st) : conflict_exact_local(p, ids, st);
}

// ================================ 2D ======================================
// predicates.hpp:337-589 (orient2d, incircle).  Bounds as the reference's
// constexpr initialisers compute them.
constexpr float kIccErrA = (float)((10.0 + 96.0 * (double)kEps) * (double)kEps);
constexpr float kCcwErrA = (float)((3.0 + 16.0 * (double)kEps) * (double)kEps);

// p.x*q.y - q.x*p.y (Two_Product, Two_Product, Two_Two_Diff).
__device__ __forceinline__ void minor2xy(const float2 p, const float2 q, float m[4]) {
    minor2(make_float3(p.x, p.y, 0.f), make_float3(q.x, q.y, 0.f), m);
}
// p*q1 - p*q2 as a 4-term expansion (the aterms / bterms of orient2dexact).
__device__ __forceinline__ void prod_diff(float p, float q1, float q2, float m[4]) {
    float h1, l1, h2, l2, i, j, z;
    two_product(p, q1, h1, l1);
    two_product(p, q2, h2, l2);
    two_diff(l1, l2, i, m[0]);
    two_sum(h1, i, j, z);
    two_diff(z, h2, i, m[1]);
    two_sum(j, i, m[3], m[2]);
}

// orient2dexact (predicates.hpp:342-383).
static __device__ __noinline__ float orient2d_exact(const float2 a, const float2 b, const float2 c, uint32_t& st) {
    float at[4], bt[4], v[8], w[12];
    prod_diff(a.x, b.y, c.y, at);
    prod_diff(b.x, c.y, a.y, bt);
    const int vl = fes(4, at, 4, bt, v, 8, st);
    prod_diff(c.x, a.y, b.y, at);
    const int wl = fes(vl, v, 4, at, w, 12, st);
    return w[wl - 1];
}

// orient2d: stage-A filter, exact when undecided (predicates.hpp:385-418).
__device__ __forceinline__ float orient2d(const float2 a, const float2 b, const float2 c, uint32_t& st) {
    const float detleft = (a.x - c.x) * (b.y - c.y);
    const float detright = (a.y - c.y) * (b.x - c.x);
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
    const float eb = kCcwErrA * detsum;
    if (det >= eb || -det >= eb) return det;
    return orient2d_exact(a, b, c, st);
}

// incircle FP32 filter (predicates.hpp:544-586) with its explicit fmaf.
__device__ __forceinline__ float incircle32(const float2 a, const float2 b, const float2 c, const float2 d,
                                            float& err) {
    const float adx = a.x - d.x, bdx = b.x - d.x, cdx = c.x - d.x;
    const float ady = a.y - d.y, bdy = b.y - d.y, cdy = c.y - d.y;
    const float bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
    const float alift = fmaf(adx, adx, ady * ady);
    const float cdxady = cdx * ady, adxcdy = adx * cdy;
    const float blift = fmaf(bdx, bdx, bdy * bdy);
    const float adxbdy = adx * bdy, bdxady = bdx * ady;
    const float clift = fmaf(cdx, cdx, cdy * cdy);
    const float det = fmaf(alift, (bdxcdy - cdxbdy), fmaf(blift, (cdxady - adxcdy), clift * (adxbdy - bdxady)));
    const float perm = fmaf(alift, (fabsf(bdxcdy) + fabsf(cdxbdy)),
                            fmaf(blift, (fabsf(cdxady) + fabsf(adxcdy)), (fabsf(adxbdy) + fabsf(bdxady)) * clift));
    err = kIccErrA * perm;
    return det;
}

// lift * m: (m * x) * (s x) + (m * y) * (s y), s = +-1 (incircleexact's adet..ddet).
__device__ __forceinline__ int lift2(const float* m, int lm, const float2 p, float s, float* out, float* d24x,
                                     float* d24y, float* d48x, float* d48y, uint32_t& st) {
    int xl = sez(lm, m, p.x, d24x, 24, st);
    xl = sez(xl, d24x, s * p.x, d48x, 48, st);
    int yl = sez(lm, m, p.y, d24y, 24, st);
    yl = sez(yl, d24y, s * p.y, d48y, 48, st);
    return fes(xl, d48x, yl, d48y, out, 96, st);
}

// incircleexact (predicates.hpp:420-542): the same expansion sequence, so the
// sign matches the reference's including any FP32 tail underflow.
static __device__ __noinline__ float incircle_exact(const float2 a, const float2 b, const float2 c, const float2 d,
                                                   uint32_t& st) {
    float ab[4], bc[4], cd[4], da[4], ac[4], bd[4];
    minor2xy(a, b, ab);
    minor2xy(b, c, bc);
    minor2xy(c, d, cd);
    minor2xy(d, a, da);
    minor2xy(a, c, ac);
    minor2xy(b, d, bd);
    float t8[8], abc[12], bcd[12], cda[12], dab[12];
    int tl = fes(4, cd, 4, da, t8, 8, st);
    const int cdal = fes(tl, t8, 4, ac, cda, 12, st);
    tl = fes(4, da, 4, ab, t8, 8, st);
    const int dabl = fes(tl, t8, 4, bd, dab, 12, st);
    for (int i = 0; i < 4; ++i) { bd[i] = -bd[i]; ac[i] = -ac[i]; }
    tl = fes(4, ab, 4, bc, t8, 8, st);
    const int abcl = fes(tl, t8, 4, ac, abc, 12, st);
    tl = fes(4, bc, 4, cd, t8, 8, st);
    const int bcdl = fes(tl, t8, 4, bd, bcd, 12, st);
    float d24x[24], d24y[24], d48x[48], d48y[48], adet[96], bdet[96], abdet[192], cddet[192], deter[384];
    const int al = lift2(bcd, bcdl, a, 1.0f, adet, d24x, d24y, d48x, d48y, st);
    const int bl = lift2(cda, cdal, b, -1.0f, bdet, d24x, d24y, d48x, d48y, st);
    const int abl = fes(al, adet, bl, bdet, abdet, 192, st);
    const int cl = lift2(dab, dabl, c, 1.0f, adet, d24x, d24y, d48x, d48y, st);
    const int dl = lift2(abc, abcl, d, -1.0f, bdet, d24x, d24y, d48x, d48y, st);
    const int cdl = fes(cl, adet, dl, bdet, cddet, 192, st);
    const int n = fes(abl, abdet, cdl, cddet, deter, 384, st);
    return deter[n - 1];
}

// The 2D star kernel's conflict decision (DirectAlphaShape2D.cpp:437-479) for
// the local triangle (p0 = star centre, p1, p2) and the inserted point p3,
// global ids i0..i3.  Returns the reference's 'det' (> 0: conflict).
static __device__ __noinline__ float incircle_sos(float2 pa, float2 pb, float2 pc, float2 pd, uint32_t i1, uint32_t i2,
                                                 uint32_t i3, uint32_t i4, float orientation, uint32_t& st) {
    bool swp = false;
#define SB_SW(x, y, px, py) { const uint32_t t_ = y; y = x; x = t_; const float2 v_ = py; py = px; px = v_; swp = !swp; }
    if (i1 > i3) SB_SW(i1, i3, pa, pc)
    if (i2 > i4) SB_SW(i2, i4, pb, pd)
    if (i1 > i2) SB_SW(i1, i2, pa, pb)
    if (i3 > i4) SB_SW(i3, i4, pc, pd)
    if (i2 > i3) SB_SW(i2, i3, pb, pc)
#undef SB_SW
    float det = incircle_exact(pa, pb, pc, pd, st);
    int depth = 0;
    while (det == 0.0f) {
        ++depth;
        if (depth == 1) det = orient2d(pb, pc, pd, st);
        else if (depth == 2) det = -orient2d(pa, pc, pd, st);
        else det = ((int)swp + (orientation < 0.0f ? 1 : 0)) == 1 ? 1.0f : -1.0f;
    }
    if (swp) det = -det;
    return det;
}

}  // namespace pred
}  // namespace sb
