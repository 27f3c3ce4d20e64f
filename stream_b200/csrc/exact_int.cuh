// Exact signs of insphere and orient3d in fixed point, for coordinates that
// are 0 or have magnitude in [2^-6, 2^18).
//
// Such a float is a multiple of 2^-29 below 2^18, so x * 2^29 is an integer
// below 2^47 and a coordinate difference one below 2^48 (int64).  The
// determinants are the stage-A expressions of the FP32 filters (Shewchuk's
// orient3d and insphere as polynomials in the differences) evaluated in
// two's-complement integers: 2x2 minors in 128 bits, everything after in 256
// bits (insphere terms stay below 2^247, orient3d below 2^147), so the sign
// is exact.  In that range the reference's FP32 expansion arithmetic is exact
// as well (no term can underflow or overflow), so both return the true sign.
// Host-compilable, so that the arithmetic can be checked against big
// integers without a GPU.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
#define SB_XHD inline
#else
#define SB_XHD __host__ __device__ __forceinline__
#endif

namespace sb {
namespace xint {

struct I256 {
    uint64_t w[4];  // two's complement, w[0] least significant
};

SB_XHD I256 from_i128(__int128 v) {
    const uint64_t s = v < 0 ? ~0ull : 0ull;
    return I256{{(uint64_t)v, (uint64_t)((unsigned __int128)v >> 64), s, s}};
}
SB_XHD I256 add(const I256& a, const I256& b) {
    I256 r;
    unsigned __int128 c = 0;
    for (int i = 0; i < 4; ++i) {
        c += (unsigned __int128)a.w[i] + b.w[i];
        r.w[i] = (uint64_t)c;
        c >>= 64;
    }
    return r;
}
SB_XHD I256 neg(const I256& a) {
    I256 r{{~a.w[0], ~a.w[1], ~a.w[2], ~a.w[3]}};
    return add(r, I256{{1u, 0u, 0u, 0u}});
}
SB_XHD I256 sub(const I256& a, const I256& b) { return add(a, neg(b)); }
SB_XHD bool negative(const I256& a) { return (int64_t)a.w[3] < 0; }
SB_XHD int sign(const I256& a) {
    if (negative(a)) return -1;
    return (a.w[0] | a.w[1] | a.w[2] | a.w[3]) ? 1 : 0;
}
// Product modulo 2^256 (exact when the true product fits in 255 bits).
SB_XHD I256 mul(I256 a, I256 b) {
    const bool na = negative(a), nb = negative(b);
    if (na) a = neg(a);
    if (nb) b = neg(b);
    uint64_t r[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) {
        if (a.w[i] == 0) continue;
        unsigned __int128 c = 0;
        for (int j = 0; i + j < 4; ++j) {
            c += (unsigned __int128)a.w[i] * b.w[j] + r[i + j];
            r[i + j] = (uint64_t)c;
            c >>= 64;
        }
    }
    const I256 p{{r[0], r[1], r[2], r[3]}};
    return na != nb ? neg(p) : p;
}
SB_XHD I256 mul(__int128 a, const I256& b) { return mul(from_i128(a), b); }

SB_XHD bool coord_ok(float x) {
    const float ax = x < 0.0f ? -x : x;
    return x == 0.0f || (ax >= 0.015625f && ax < 262144.0f);
}
SB_XHD int64_t fixed(float x) { return (int64_t)((double)x * 536870912.0); }  // x * 2^29, exact in range

// Shewchuk's orient3d(a, b, c, d) = det[a - d; b - d; c - d].
SB_XHD int orient3d_sign(float ax, float ay, float az, float bx, float by, float bz, float cx, float cy, float cz,
                         float dx, float dy, float dz) {
    const int64_t adx = fixed(ax) - fixed(dx), bdx = fixed(bx) - fixed(dx), cdx = fixed(cx) - fixed(dx);
    const int64_t ady = fixed(ay) - fixed(dy), bdy = fixed(by) - fixed(dy), cdy = fixed(cy) - fixed(dy);
    const int64_t adz = fixed(az) - fixed(dz), bdz = fixed(bz) - fixed(dz), cdz = fixed(cz) - fixed(dz);
    const __int128 m1 = (__int128)bdx * cdy - (__int128)cdx * bdy;
    const __int128 m2 = (__int128)cdx * ady - (__int128)adx * cdy;
    const __int128 m3 = (__int128)adx * bdy - (__int128)bdx * ady;
    I256 det = mul((__int128)adz, from_i128(m1));
    det = add(det, mul((__int128)bdz, from_i128(m2)));
    det = add(det, mul((__int128)cdz, from_i128(m3)));
    return sign(det);
}

// Shewchuk's insphere(a, b, c, d, e): the lifted 4x4 determinant of the
// differences to e, in the stage-A expression's terms.
SB_XHD int insphere_sign(const float* a, const float* b, const float* c, const float* d, const float* e) {
    const int64_t aex = fixed(a[0]) - fixed(e[0]), bex = fixed(b[0]) - fixed(e[0]);
    const int64_t cex = fixed(c[0]) - fixed(e[0]), dex = fixed(d[0]) - fixed(e[0]);
    const int64_t aey = fixed(a[1]) - fixed(e[1]), bey = fixed(b[1]) - fixed(e[1]);
    const int64_t cey = fixed(c[1]) - fixed(e[1]), dey = fixed(d[1]) - fixed(e[1]);
    const int64_t aez = fixed(a[2]) - fixed(e[2]), bez = fixed(b[2]) - fixed(e[2]);
    const int64_t cez = fixed(c[2]) - fixed(e[2]), dez = fixed(d[2]) - fixed(e[2]);
    const __int128 ab = (__int128)aex * bey - (__int128)bex * aey;
    const __int128 bc = (__int128)bex * cey - (__int128)cex * bey;
    const __int128 cd = (__int128)cex * dey - (__int128)dex * cey;
    const __int128 da = (__int128)dex * aey - (__int128)aex * dey;
    const __int128 ac = (__int128)aex * cey - (__int128)cex * aey;
    const __int128 bd = (__int128)bex * dey - (__int128)dex * bey;
    const I256 abc = add(sub(mul((__int128)aez, from_i128(bc)), mul((__int128)bez, from_i128(ac))),
                         mul((__int128)cez, from_i128(ab)));
    const I256 bcd = add(sub(mul((__int128)bez, from_i128(cd)), mul((__int128)cez, from_i128(bd))),
                         mul((__int128)dez, from_i128(bc)));
    const I256 cda = add(add(mul((__int128)cez, from_i128(da)), mul((__int128)dez, from_i128(ac))),
                         mul((__int128)aez, from_i128(cd)));
    const I256 dab = add(add(mul((__int128)dez, from_i128(ab)), mul((__int128)aez, from_i128(bd))),
                         mul((__int128)bez, from_i128(da)));
    const __int128 alift = (__int128)aex * aex + (__int128)aey * aey + (__int128)aez * aez;
    const __int128 blift = (__int128)bex * bex + (__int128)bey * bey + (__int128)bez * bez;
    const __int128 clift = (__int128)cex * cex + (__int128)cey * cey + (__int128)cez * cez;
    const __int128 dlift = (__int128)dex * dex + (__int128)dey * dey + (__int128)dez * dez;
    const I256 det = add(sub(mul(dlift, abc), mul(clift, dab)), sub(mul(blift, cda), mul(alift, bcd)));
    return sign(det);
}

}  // namespace xint
}  // namespace sb
