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


# ---- 2D alpha shape (src/mesh/DirectAlphaShape2D.cpp) -------------------------
_AS2_KEYS = ("perm", "elems", "row", "neig", "edge_is_bnd", "node_is_bnd", "nineig", "nelem")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ashape2d_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_restatement_matches_golden_ashape2d(restate, path):
    g = np.load(path)
    r = restate.ashape2d(g["pts"], g["alpha"])
    for k in _AS2_KEYS:
        assert np.array_equal(getattr(r, k), g[k]), k


def _cases2d():
    from stream_b200 import workloads
    rng = np.random.default_rng(3)
    u = rng.random((3000, 2)).astype(np.float32)
    circ = np.stack([np.cos(np.arange(300) * (2 * np.pi / 300)), np.sin(np.arange(300) * (2 * np.pi / 300))], 1)
    return {
        "lattice_fill_limit": workloads.lattice2d(40, alpha=0.2),  # stars stop at the 250-id limit
        "duplicates": (np.concatenate([u, u[:400]]), np.full(3400, 0.04, np.float32)),
        "cocircular": (np.concatenate([circ, [[0.0, 0.0]]]).astype(np.float32), np.full(301, 0.5, np.float32)),
        "collinear": (np.stack([np.linspace(0, 1, 200), np.zeros(200)], 1).astype(np.float32),
                      np.full(200, 0.02, np.float32)),
        "tiny_coords": ((rng.random((1500, 2)) * 1e-6).astype(np.float32), np.full(1500, 1e-7, np.float32)),
        "variable_alpha": (u, (rng.random(3000) * 0.05 + 0.005).astype(np.float32)),
    }


@pytest.mark.parametrize("case", list(_cases2d().keys()))
def test_restatement_vs_reference_build_ashape2d(restate, reference, case):
    pts, al = _cases2d()[case]
    a, b = restate.ashape2d(pts, al), reference.ashape2d(pts, al)
    for k in _AS2_KEYS + ("coords_m", "cand", "bb_glob", "morton"):
        x, y = getattr(a, k), getattr(b, k)
        assert x.shape == y.shape and np.array_equal(x, y), k


def test_ashape2d_published_triangle_count(restate):
    """testcases/IMR26/README.md:48-54: uniform2D -n 1000000 -a 0.0012 (glibc
    srand(42) stream) gives 1,877,465 triangles."""
    from stream_b200 import workloads
    pts, al = workloads.glibc_uniform_square(1_000_000, 0.0012)
    r = restate.ashape2d(pts, al)
    assert r.status == 0
    assert len(r.elems) == 1_877_465


def test_predicates2d_exact_signs(restate):
    """orient2d / incircle exact signs against rational arithmetic on random,
    co-circular and collinear quadruples (predicates.hpp:337-589)."""
    from fractions import Fraction
    import ctypes
    L = restate.lib
    L.orc_incircle_exact.restype = ctypes.c_float
    L.orc_orient2d.restype = ctypes.c_float
    rng = np.random.default_rng(5)
    quads = [rng.random((4, 2)).astype(np.float32) for _ in range(200)]
    quads += [np.array([[0, 0], [1, 0], [0, 1], [1, 1]], np.float32)]          # co-circular
    quads += [np.array([[0, 0], [1, 1], [2, 2], [0.5, 3]], np.float32)]        # collinear a, b, c
    quads += [(np.array([[0, 0], [1, 0], [0, 1], [1, 1]]) * 1e-5 + 0.3).astype(np.float32)]

    def sgn(v):
        return (v > 0) - (v < 0)

    for q in quads:
        F = [[Fraction(float(v)) for v in p] for p in q]
        a, b, c, d = F
        o = (a[0] - c[0]) * (b[1] - c[1]) - (a[1] - c[1]) * (b[0] - c[0])
        m = [[p[0] - d[0], p[1] - d[1], (p[0] - d[0]) ** 2 + (p[1] - d[1]) ** 2] for p in (a, b, c)]
        ic = (m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2]) - m[0][1] * (m[1][0] * m[2][2] - m[2][0] * m[1][2])
              + m[0][2] * (m[1][0] * m[2][1] - m[2][0] * m[1][1]))
        p = [np.ascontiguousarray(v).ctypes.data_as(ctypes.c_void_p) for v in q]
        assert sgn(L.orc_orient2d(p[0], p[1], p[2])) == sgn(o)
        assert sgn(L.orc_incircle_exact(*p)) == sgn(ic)


def test_restatement_vs_reference_build_ashape2d_glibc_100k(restate, reference):
    """uniform2D -n 100000 -a 0.006 (a size of testcases/IMR26/README.md:34-41):
    every output of the restatement equals the reference build's."""
    from stream_b200 import workloads
    pts, al = workloads.glibc_uniform_square(100_000, 0.006)
    a, b = restate.ashape2d(pts, al), reference.ashape2d(pts, al)
    for k in _AS2_KEYS + ("coords_m", "cand", "bb_glob", "morton"):
        x, y = getattr(a, k), getattr(b, k)
        assert x.shape == y.shape and np.array_equal(x, y), k


def test_restatement_ashape2d_thread_count_independent():
    """The 2D restatement's outputs do not depend on the OpenMP thread count
    (each point's star is computed alone; scans are sequential)."""
    import subprocess
    import sys
    code = ("import sys, numpy as np; sys.path.insert(0, '.');"
            "from oracle.oracle import Restatement; from stream_b200 import workloads;"
            "p, a = workloads.uniform_square(20000, seed=9); r = Restatement().ashape2d(p, a);"
            "import hashlib; print(hashlib.sha256(r.elems.tobytes() + r.neig.tobytes() + r.perm.tobytes()).hexdigest())")
    outs = {subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True,
                           cwd=os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                           env=dict(os.environ, OMP_NUM_THREADS=str(t))).stdout.strip() for t in (1, 4)}
    assert len(outs) == 1, outs


# ---- TRBVH treelet restructuring (include/geometry/trbvh.hpp:392-679) ---------
_TR_KEYS = ("child_left", "child_right", "range_min", "range_max", "parent", "bboxes", "subtree_size", "sah",
            "obj_m", "root")


def _tr_same(a, b):
    for k in _TR_KEYS:
        x, y = np.atleast_1d(np.asarray(a[k])), np.atleast_1d(np.asarray(b[k]))
        assert x.shape == y.shape and np.array_equal(x.view(np.uint8), y.view(np.uint8)), k


def _lbvha_of_restatement(restate, xyzr):
    t = restate.trbvh3d(xyzr, treelet_size=5, area3d=False, rounds=0)
    return dict(children=np.stack([t["child_left"], t["child_right"]], 1),
                range=np.stack([t["range_min"], t["range_max"]], 1), parent=t["parent"], bboxes=t["bboxes"],
                root=t["root"], obj_m=t["obj_m"])


def test_restatement_matches_golden_lbvha(restate):
    """The reference's LBVHa (include/geometry/lbvh_agglo.hpp:270-325) is the
    Apetrei build the TRBVH starts from: same children, ranges, parents and
    boxes (boxes combine exactly, so arrival order does not matter)."""
    g = np.load(os.path.join(GOLDEN, "lbvha_uniform_1500.npz"))
    got = _lbvha_of_restatement(restate, g["xyzr"])
    for k in ("children", "range", "parent", "bboxes", "root", "obj_m"):
        assert np.array_equal(np.atleast_1d(got[k]).view(np.uint8), np.atleast_1d(g[k]).view(np.uint8)), k


@pytest.mark.parametrize("n", [2, 5, 20_000, 100_003])
def test_restatement_vs_reference_build_lbvha(restate, reference, n):
    rng = np.random.default_rng(n)
    xyzr = np.concatenate([rng.random((n, 3)), 0.01 * (1 + rng.random((n, 1)))], 1).astype(np.float32)
    got, want = _lbvha_of_restatement(restate, xyzr), reference.lbvha3d(xyzr)
    for k in want:
        assert np.array_equal(np.atleast_1d(got[k]).view(np.uint8), np.atleast_1d(want[k]).view(np.uint8)), k


def test_restatement_matches_golden_trbvh(restate):
    """The reference's full TRBVH build (Apetrei build + three rounds of
    5-leaf treelet restructuring, 2D SAH area) on spheres of radius 0, where
    its order-dependent SAH sums coincide with the restatement's fixed order."""
    g = np.load(os.path.join(GOLDEN, "trbvh_r0_2000.npz"))
    _tr_same(restate.trbvh3d(g["xyzr"], treelet_size=5, area3d=False, rounds=3), g)


@pytest.mark.parametrize("n,seed", [(5, 0), (64, 1), (1000, 2), (20_000, 3)])
def test_restatement_vs_reference_build_trbvh(restate, reference, n, seed):
    rng = np.random.default_rng(seed)
    xyzr = np.concatenate([rng.random((n, 3)), np.zeros((n, 1))], 1).astype(np.float32)
    _tr_same(restate.trbvh3d(xyzr, treelet_size=5, area3d=False, rounds=3),
             reference.trbvh3d(xyzr, optimize=True, threads=1))


# ---- full-size fixtures (tests/golden/digests.json) -----------------------------
def _digest_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("_golden_digest", os.path.join(GOLDEN, "digest.py"))
    dg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(dg)
    return dg


@pytest.mark.parametrize("case", ["uniform3d_100000_0.022", "uniform3d_50000_0.036"])
def test_restatement_matches_reference_digests_uniform3d(restate, case):
    """The reference's uniform3D cloud (glibc srand(42)) and its published
    example (100,000 points, alpha 0.022: 526,040 tets on the author's GPU,
    testcases/IMR26/README.md:93-99; 526,042 from its sources built without
    FMA contraction): the restatement reproduces the reference build's
    outputs digest for digest."""
    import json
    from stream_b200 import workloads
    dg = _digest_module()
    rec = json.load(open(os.path.join(GOLDEN, "digests.json")))[case]
    pts, al = workloads.glibc_uniform_cube(rec["points"], rec["alpha"])
    assert dg.input_digest(pts, al) == rec["input"]
    got = dg.mesh_digests(dg.mesh_arrays_from_result(restate.ashape3d(pts, al)))
    assert got == {k: rec["mesh"][k] for k in got}


def test_restatement_matches_reference_digests_stress_subcube(restate):
    """The 223,766-point corner of the 4M meshing-stress cloud (blobs with
    truncated stars, lattice sites, uniform points): restatement = reference
    build, digest for digest."""
    import json
    from stream_b200 import workloads
    dg = _digest_module()
    rec = json.load(open(os.path.join(GOLDEN, "digests.json")))["stress_subcube"]
    pts, al, _ = workloads.sub_cube(*workloads.meshing_stress(4_000_000, seed=0), 200_000)
    assert dg.input_digest(pts, al) == rec["input"]
    got = dg.mesh_digests(dg.mesh_arrays_from_result(restate.ashape3d(pts, al)))
    assert got == {k: rec["mesh"][k] for k in got}


def test_deep_tree_restatement_vs_reference_build(restate, reference):
    """Point pairs converging on one point with a search radius that reaches
    them all (workloads.deep_spine, distinct Morton codes): every LBVH array and
    every mesh output of the restatement equals the reference build's, with
    no traversal-stack overflow."""
    from stream_b200 import workloads
    pts, al = workloads.deep_spine()
    xyzr = np.concatenate([pts, al[:, None]], 1)
    assert len(np.unique(restate.lbvh3d(xyzr)["morton"])) == len(pts)
    ta, tb = restate.lbvh3d(xyzr), reference.lbvh3d(xyzr)
    for k in ta:
        assert np.array_equal(ta[k].view(np.uint8), tb[k].view(np.uint8)), k
    a, b = restate.ashape3d(pts, al), reference.ashape3d(pts, al)
    assert not (a.status & 1)
    for k in ("perm", "elems", "row", "neig", "edge_is_bnd", "node_is_bnd", "nineig", "nelem"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
