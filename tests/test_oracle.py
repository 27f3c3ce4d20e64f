"""CPU: the oracle restatement pinned against the reference's own outputs
(golden fixtures made by tests/golden/make_golden.py from the reference
sources) and against the reference build when present; known answers of the
reference's tests."""
import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _ashape_fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "ashape_*.npz")))


@pytest.mark.parametrize("path", _ashape_fixtures(), ids=lambda p: os.path.basename(p))
def test_restatement_matches_golden_ashape(restate, path):
    g = np.load(path)
    r = restate.ashape3d(g["pts"], g["alpha"])
    for k in ("perm", "elems", "row", "neig", "edge_is_bnd", "node_is_bnd", "nineig"):
        assert np.array_equal(getattr(r, k), g[k]), k


def test_restatement_matches_golden_lbvh(restate):
    g = np.load(os.path.join(GOLDEN, "lbvh_uniform_1500.npz"))
    r = restate.lbvh3d(g["xyzr"])
    for k in ("bb_glob", "morton", "perm", "sep", "cil", "leaf_parent", "internal_parent", "bboxes", "obj_m"):
        assert np.array_equal(r[k].view(np.uint8), g[k].view(np.uint8)), k


@pytest.mark.parametrize("n", [2, 5, 64, 3000])
def test_restatement_vs_reference_build_lbvh(restate, reference, n):
    rng = np.random.default_rng(n)
    xyzr = np.concatenate([rng.random((n, 3)), rng.random((n, 1)) * 0.05], 1).astype(np.float32)
    a, b = restate.lbvh3d(xyzr), reference.lbvh3d(xyzr)
    for k in a:
        assert np.array_equal(a[k].view(np.uint8), b[k].view(np.uint8)), k


def test_restatement_vs_reference_build_ashape_mixed(restate, reference):
    from stream_b200 import workloads
    pts, al = workloads.meshing_stress(8000, seed=1)
    a, b = restate.ashape3d(pts, al), reference.ashape3d(pts, al)
    for k in ("perm", "elems", "row", "neig", "edge_is_bnd", "node_is_bnd", "nineig", "nelem"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_lbvh_line_kat(restate):
    """tests/geometry/lbvh_simple_collision.cpp:83-86 (lifted to 3D): spheres of
    radius 0.55 on a line give the root box [-0.55, n-1+0.55] x [-0.55, 0.55]^2."""
    n = 100
    xyzr = np.zeros((n, 4), np.float32)
    xyzr[:, 0] = np.arange(n)
    xyzr[:, 3] = 0.55
    root = restate.lbvh3d(xyzr)["bboxes"][0]
    f = np.float32
    assert root.tolist() == [f(-0.55), f(-0.55), f(-0.55), f(n - 1) + f(0.55), f(0.55), f(0.55)]


def test_cg_diagonal_kat(restate):
    """tests/numerics/cg_jacobi.cpp:36-83: diag(1..100) x = 1 -> x_i = 1/i."""
    n = 100
    row = np.arange(n + 1, dtype=np.uint32)
    x, it = restate.cg_f32(row, row[:-1], np.arange(1, n + 1, dtype=np.float32), np.ones(n, np.float32),
                           np.zeros(n, np.float32))
    assert np.max(np.abs(x - 1.0 / np.arange(1, n + 1))) <= 1e-7


def test_predicates_known_signs(restate):
    """insphere/orient3d sign conventions and the SoS tie-break on a
    co-spherical configuration (DirectAlphaShape3D.cpp:442-480)."""
    # e strictly inside / outside the unit-cube circumsphere of (a,b,c,d)
    cube = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
    inside = np.concatenate([cube, [[0.5, 0.5, 0.5]]]).astype(np.float32)
    outside = np.concatenate([cube, [[3, 3, 3]]]).astype(np.float32)
    cosph = np.concatenate([cube, [[1, 1, 1]]]).astype(np.float32)
    ids = np.array([[0, 1, 2, 3, 4]] * 3, np.uint32)
    det, used = restate.conflict_batch(np.stack([inside, outside, cosph]), ids)
    # orientation of (a,b,c,d) decides the sign convention; inside/outside differ
    assert np.sign(det[0]) == -np.sign(det[1]) and det[0] != 0 and det[1] != 0
    assert used[2] == 1 and det[2] != 0  # exactly co-spherical: exact stage + SoS
