"""LBVH on the GPU vs the oracle: bit-exact global box, Morton codes, sort
permutation, Karras topology and node boxes (include/geometry/lbvh.hpp)."""
import numpy as np
import pytest

from stream_b200 import workloads

pytestmark = pytest.mark.gpu

KEYS = ("bb_glob", "morton", "perm", "sep", "cil", "leaf_parent", "internal_parent", "bboxes", "obj_m")


def _xyzr(pts, r):
    return np.concatenate([pts, np.broadcast_to(np.float32(r), (len(pts), 1))], axis=1).astype(np.float32)


def _check(sb, restate, xyzr, bits=63, fit_point=False):
    from stream_b200.geometry import Sphere3DLBVH
    b = Sphere3DLBVH()
    b.set_objects(xyzr, bits=bits, fit_point=fit_point)
    st = b.build()
    assert st == 0, f"status 0x{st:x}"
    got = b.arrays()
    want = restate.lbvh3d(xyzr, bits=bits, fit_point=fit_point)
    for k in KEYS:
        assert got[k].shape == want[k].shape, k
        assert np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)), f"{k} differs"


@pytest.mark.parametrize("n", [2, 3, 17, 1000, 4096, 4097, 100_003])
@pytest.mark.parametrize("bits", [63, 30])
def test_lbvh_uniform(sb, restate, n, bits):
    pts, _ = workloads.uniform_cube(n, seed=n)
    _check(sb, restate, _xyzr(pts, 0.01), bits=bits)


@pytest.mark.parametrize("fit_point", [False, True])
def test_lbvh_mixed_cloud(sb, restate, fit_point):
    pts, a = workloads.meshing_stress(50_000, seed=3)
    _check(sb, restate, _xyzr(pts, a[0]), fit_point=fit_point)


def test_lbvh_duplicates_and_lattice(sb, restate):
    pts, _ = workloads.lattice(12)
    pts = np.concatenate([pts, pts[:300]])  # exact duplicates: equal Morton codes
    _check(sb, restate, _xyzr(pts, 0.02))


def test_lbvh_line_kat(sb, restate):
    # Known answer of tests/geometry/lbvh_simple_collision.cpp:83-86, lifted to 3D:
    # spheres of radius 0.55 at x = 0..n-1 -> root box [-0.55, n-1+0.55] x [-0.55, 0.55]^2.
    from stream_b200.geometry import Sphere3DLBVH
    n = 100
    xyzr = np.zeros((n, 4), np.float32)
    xyzr[:, 0] = np.arange(n)
    xyzr[:, 3] = 0.55
    b = Sphere3DLBVH()
    b.set_objects(xyzr)
    assert b.build() == 0
    root = b.arrays()["bboxes"][0]
    assert root.tolist() == [np.float32(-0.55), np.float32(-0.55), np.float32(-0.55),
                             np.float32(n - 1) + np.float32(0.55), np.float32(0.55), np.float32(0.55)]


@pytest.mark.slow
def test_lbvh_4m_properties(sb):
    """Full-size meshing-stress cloud: sortedness, stable permutation and a
    consistent tree (every non-root node has exactly one parent that names it)."""
    from stream_b200.geometry import Sphere3DLBVH
    pts, a = workloads.meshing_stress(4_000_000, seed=0)
    xyzr = _xyzr(pts, a[0])
    b = Sphere3DLBVH()
    b.set_objects(xyzr)
    assert b.build() == 0
    g = b.arrays()
    m, perm = g["morton"], g["perm"]
    assert np.all(m[1:] >= m[:-1])
    assert np.array_equal(np.sort(perm), np.arange(len(perm), dtype=np.uint32))
    ties = m[1:] == m[:-1]
    assert np.all(perm[1:][ties] > perm[:-1][ties])  # stability
    n = len(perm)
    sep, cil = g["sep"].astype(np.int64), g["cil"]
    left_leaf = (cil & 1) != 0
    right_leaf = (cil & 2) != 0
    leaves = np.concatenate([sep[left_leaf], sep[right_leaf] + 1])
    internals = np.concatenate([sep[~left_leaf], sep[~right_leaf] + 1])
    assert np.array_equal(np.sort(leaves), np.arange(n))
    assert np.array_equal(np.sort(internals), np.arange(1, n - 1))
    # Root box contains every object.
    root = g["bboxes"][0]
    assert np.all(xyzr[:, :3] - xyzr[:, 3:] >= root[:3]) and np.all(xyzr[:, :3] + xyzr[:, 3:] <= root[3:])
