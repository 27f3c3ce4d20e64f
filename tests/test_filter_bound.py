"""The per-star bound of the FP32 insphere filter's error bound
(star_filter_bound in stream_b200/csrc/predicates.cuh): for five points
within mc of the star centre in each coordinate, the filter's
err = kIspErrA x permanent, evaluated in FP32 with the filter's operations,
never exceeds the bound, so a test whose |det| is above the bound is certain
under the filter with the same det.  Restated in numpy (FP32 steps, fmaf as
an exactly rounded double expression) over random and worst-case (every
difference at 2 mc) configurations from mc = 2^-21 to just below 2^19."""
import numpy as np

F = np.float32
EPS = 2.0 ** -24
ISP_ERR_A = F((16.0 + 224.0 * EPS) * EPS)


def star_filter_bound(mc):
    """The CUDA function, element-wise (INFINITY outside [2^-21, 2^19))."""
    mc = np.asarray(mc, np.float32)
    D = 2.0 * mc.astype(np.float64) * (1.0 + 2.0 ** -20)
    b = float(ISP_ERR_A) * 72.0 * D ** 5 * (1.0 + 2.0 ** -16) + 2.0 ** -120
    bf = b.astype(np.float32)
    bf = np.where(bf.astype(np.float64) < b, np.nextafter(bf, np.float32(np.inf)), bf)  # round up
    ok = (mc >= F(2.0 ** -21)) & (mc < F(2.0 ** 19))
    return np.where(ok, bf, np.float32(np.inf))


def fmaf(a, b, c):
    return (a.astype(np.float64) * b.astype(np.float64) + c.astype(np.float64)).astype(np.float32)


def filter_err(a, b, c, d, e):
    """kIspErrA x permanent of the FP32 filter (predicates.hpp:986-1100), arrays (m, 3)."""
    aex, aey, aez = (F(0) + a - e).T
    bex, bey, bez = (b - e).T
    cex, cey, cez = (c - e).T
    dex, dey, dez = (d - e).T
    ab = lambda x, y: np.abs(x * y)  # noqa: E731  float32 product
    aexbey, bexaey, bexcey, cexbey = ab(aex, bey), ab(bex, aey), ab(bex, cey), ab(cex, bey)
    cexdey, dexcey, dexaey, aexdey = ab(cex, dey), ab(dex, cey), ab(dex, aey), ab(aex, dey)
    aexcey, cexaey, bexdey, dexbey = ab(aex, cey), ab(cex, aey), ab(bex, dey), ab(dex, bey)
    lift = lambda x, y, z: fmaf(x, x, fmaf(y, y, z * z))  # noqa: E731
    alift, blift, clift, dlift = lift(aex, aey, aez), lift(bex, bey, bez), lift(cex, cey, cez), lift(dex, dey, dez)
    az, bz, cz, dz = np.abs(aez), np.abs(bez), np.abs(cez), np.abs(dez)
    ta = fmaf(bz, cexdey + dexcey, fmaf(cz, dexbey + bexdey, dz * (bexcey + cexbey)))
    tb = fmaf(cz, dexaey + aexdey, fmaf(dz, aexcey + cexaey, az * (cexdey + dexcey)))
    tc = fmaf(dz, aexbey + bexaey, fmaf(az, bexdey + dexbey, bz * (dexaey + aexdey)))
    td = fmaf(az, bexcey + cexbey, fmaf(bz, cexaey + aexcey, cz * (aexbey + bexaey)))
    perm = fmaf(alift, ta, fmaf(blift, tb, fmaf(clift, tc, dlift * td)))
    return ISP_ERR_A * perm


def _case(rng, m, mc, centre_scale, worst):
    centre = (rng.uniform(-1, 1, (m, 3)) * centre_scale).astype(np.float32)
    if worst:  # a, b, c, d at +mc, e at -mc in every coordinate: the largest permanent, 72 (2 mc)^5
        u = np.concatenate([np.ones((4, m, 3)), -np.ones((1, m, 3))])
    else:
        u = rng.uniform(-1, 1, (5, m, 3))
    pts = (centre[None] + (u * mc).astype(np.float32)).astype(np.float32)
    # the kernel's mc: the rounded maximum offset of the star's points from the centre
    mck = np.abs(pts - centre[None]).astype(np.float32).max(axis=(0, 2))
    return pts, mck


def test_bound_covers_filter_error():
    rng = np.random.default_rng(7)
    m = 20000
    for k in (-20.9, -17, -12, -6, -1, 0, 3, 9, 15, 18.9):
        mc = 2.0 ** k
        for centre_scale in (0.0, mc, 1.0, 1000.0):
            for worst in (False, True):
                pts, mck = _case(rng, m, mc, centre_scale, worst)
                bound = star_filter_bound(mck)
                err = filter_err(*pts)
                finite = np.isfinite(bound)
                if centre_scale * 2.0 ** -20 < mc:  # offsets resolvable at the centre's magnitude
                    assert finite.any(), (k, centre_scale, worst)
                assert np.all(err[finite] <= bound[finite]), (k, centre_scale, worst)
                if worst and centre_scale == 0.0:  # every offset exactly +-mc: the bound is tight there
                    assert np.all(bound[finite] <= 1.001 * err[finite] + 2.0 ** -119), k


def test_bound_off_outside_its_range():
    assert np.isinf(star_filter_bound(np.float32(0.0)))
    assert np.isinf(star_filter_bound(np.float32(2.0 ** -22)))
    assert np.isinf(star_filter_bound(np.float32(2.0 ** 19)))
    assert np.isinf(star_filter_bound(np.float32(np.inf)))
    assert np.isinf(star_filter_bound(np.float32(np.nan)))
    assert np.isfinite(star_filter_bound(np.float32(2.0 ** -21)))
