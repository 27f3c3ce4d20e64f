"""Seeded synthetic point clouds of the benchmark configurations.

No public dataset is involved; these generators stand in for the shapes the
benchmark names.  Coordinates are drawn in FP64 and rounded to FP32 (the
mesher's input type, as in the reference, where fp_tt is float).
"""
from __future__ import annotations

import numpy as np


def uniform_cube(n: int, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """n points uniform in [0,1)^3, alpha = 1.3 * n^(-1/3) (the 200k plain-method case)."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 3)).astype(np.float32)
    alpha = np.full(n, 1.3 * n ** (-1.0 / 3.0), dtype=np.float32)
    return pts, alpha


def meshing_stress(n: int = 4_000_000, seed: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """60% uniform in the unit cube, 30% in 32 isotropic Gaussian blobs
    (sigma 0.01, centres uniform, not clipped) and 10% distinct sites of the
    100^3 integer lattice scaled to [0,1]^3 (k/99); alpha = 1.5 * n^(-1/3)."""
    rng = np.random.default_rng(seed)
    n_uni = int(round(0.6 * n))
    n_lat = int(round(0.1 * n))
    n_blob = n - n_uni - n_lat
    uni = rng.random((n_uni, 3))
    centres = rng.random((32, 3))
    which = rng.integers(0, 32, size=n_blob)
    blob = centres[which] + 0.01 * rng.standard_normal((n_blob, 3))
    sites = rng.choice(100 ** 3, size=min(n_lat, 100 ** 3), replace=False)
    lat = np.stack([sites // 10000, (sites // 100) % 100, sites % 100], axis=1) / 99.0
    pts = np.concatenate([uni, blob, lat]).astype(np.float32)
    perm = rng.permutation(n)
    pts = np.ascontiguousarray(pts[perm])
    alpha = np.full(n, 1.5 * n ** (-1.0 / 3.0), dtype=np.float32)
    return pts, alpha


def sub_cube(pts: np.ndarray, alpha: np.ndarray, target: int) -> tuple[np.ndarray, np.ndarray, float]:
    """The points of the smallest corner box [lo, lo + s (hi - lo)] (s on a
    grid of 33 steps from 0.2 to 1) that holds at least target points, in
    input order, with their alpha: the same local density and neighbour counts
    as the whole cloud.  Returns (points, alpha, s)."""
    lo = pts.min(axis=0)
    hi = pts.max(axis=0)
    for s in np.linspace(0.2, 1.0, 33):
        box_hi = lo + s * (hi - lo)
        m = np.all(pts <= box_hi, axis=1)
        if m.sum() >= target:
            return np.ascontiguousarray(pts[m]), np.ascontiguousarray(alpha[m]), float(s)
    return pts, alpha, 1.0


def dambreak_column(h: float = 0.01, seed: int = 0, extent=(0.4, 0.8, 0.4)) -> tuple[np.ndarray, np.ndarray]:
    """Jittered lattice of spacing h filling a 0.4 x 0.8 x 0.4 column, jitter
    uniform in +-0.1h per axis, alpha = 1.2h."""
    rng = np.random.default_rng(seed)
    m = [int(round(e / h)) for e in extent]
    g = np.stack(np.meshgrid(*[np.arange(k) for k in m], indexing="ij"), -1).reshape(-1, 3)
    pts = (g + 0.5) * h + rng.uniform(-0.1 * h, 0.1 * h, size=g.shape)
    pts = pts.astype(np.float32)
    alpha = np.full(len(pts), 1.2 * h, dtype=np.float32)
    return pts, alpha


def deep_spine(levels: int = 50, alpha: float = 0.6) -> tuple[np.ndarray, np.ndarray]:
    """Pairs of points converging on (0.9, 0.9, 0.9), each pair 2^(1/3) times
    closer than the one before, with a search radius that reaches every
    point: each level shares more Morton bits with the limit point, so the
    LBVH is deep and every internal node is visited.  The 2 * levels points
    keep distinct 63-bit Morton codes (the reference's hierarchy has no index
    tie-break, so duplicate codes leave it ill-defined)."""
    P = np.array([0.9, 0.9, 0.9])
    pts = []
    for j in range(levels):
        q = P - 2.0 ** (-j / 3.0) * np.array([0.5, 0.5, 0.5])
        pts += [q, q + np.array([0.0, 0.0, 2.0 ** -19])]
    pts = np.array(pts, np.float32)
    return pts, np.full(len(pts), alpha, dtype=np.float32)


def lattice(m: int, spacing: float | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Full m^3 lattice k/(m-1) (maximal co-spherical degeneracy)."""
    g = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3) / float(m - 1)
    pts = g.astype(np.float32)
    a = 1.5 / (m - 1) if spacing is None else spacing
    return pts, np.full(len(pts), a, dtype=np.float32)


# ---- 2D --------------------------------------------------------------------
def uniform_square(n: int, seed: int = 0, alpha: float | None = None) -> tuple[np.ndarray, np.ndarray]:
    """n points uniform in [0,1)^2, alpha = 1.2 * n^(-1/2) unless given."""
    rng = np.random.default_rng(seed)
    pts = rng.random((n, 2)).astype(np.float32)
    a = 1.2 * n ** -0.5 if alpha is None else alpha
    return pts, np.full(n, a, dtype=np.float32)


def glibc_uniform_square(n: int, alpha: float, seed: int = 42) -> tuple[np.ndarray, np.ndarray]:
    """The reference's uniform2D benchmark cloud: glibc srand(seed), then
    x = (float) rand() / RAND_MAX, y likewise, per point
    (testcases/IMR26/uniform2D.cpp:130-142).  The C library's rand() is called
    through ctypes, so the stream is the one the reference's harness draws on
    this platform."""
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(seed))
    rnd = libc.rand
    vals = np.fromiter((rnd() for _ in range(2 * n)), dtype=np.float32, count=2 * n)
    pts = (vals / np.float32(2147483647)).astype(np.float32).reshape(n, 2)
    return pts, np.full(n, alpha, dtype=np.float32)


def glibc_uniform_cube(n: int, alpha: float, seed: int = 42) -> tuple[np.ndarray, np.ndarray]:
    """The reference's uniform3D benchmark cloud: glibc srand(seed), then for
    each point x, y, z = (float) rand() / RAND_MAX in that order
    (testcases/IMR26/uniform3D.cpp:130-142).  The C library's rand() is
    called through ctypes, so the stream is the one the reference's harness
    draws on this platform; RAND_MAX converted to float is 2^31."""
    import ctypes
    libc = ctypes.CDLL("libc.so.6")
    libc.srand(ctypes.c_uint(seed))
    rnd = libc.rand
    vals = np.fromiter((rnd() for _ in range(3 * n)), dtype=np.float32, count=3 * n)
    pts = (vals / np.float32(2147483647)).astype(np.float32).reshape(n, 3)
    return pts, np.full(n, alpha, dtype=np.float32)


# The paper's uniform3D sweep, (points, alpha) (testcases/IMR26/README.md:80-86).
UNIFORM3D_SWEEP = ((10_000, 0.06), (50_000, 0.036), (100_000, 0.024), (500_000, 0.0144), (1_000_000, 0.0108))


def lattice2d(m: int, alpha: float | None = None) -> tuple[np.ndarray, np.ndarray]:
    """Full m x m lattice k/(m-1) (maximal co-circular degeneracy)."""
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 2) / float(m - 1)
    a = 1.5 / (m - 1) if alpha is None else alpha
    return g.astype(np.float32), np.full(m * m, a, dtype=np.float32)


def dambreak_column2d(h: float = 0.01, seed: int = 0, extent=(0.4, 0.8)) -> tuple[np.ndarray, np.ndarray]:
    """Jittered lattice of spacing h filling a 0.4 x 0.8 column, jitter uniform
    in +-0.1h per axis, alpha = 1.2h."""
    rng = np.random.default_rng(seed)
    m = [int(round(e / h)) for e in extent]
    g = np.stack(np.meshgrid(*[np.arange(k) for k in m], indexing="ij"), -1).reshape(-1, 2)
    pts = ((g + 0.5) * h + rng.uniform(-0.1 * h, 0.1 * h, size=g.shape)).astype(np.float32)
    return pts, np.full(len(pts), 1.2 * h, dtype=np.float32)
