"""TRBVH on the GPU (include/geometry/trbvh.hpp): the Apetrei build equals the
reference's topology, ranges, boxes and subtree sizes; the restructured tree
equals the reference build's on zero-radius spheres (where the reference's
SAH sums are deterministic) and the oracle's everywhere (order-independent
SAH); queries through it find exactly the overlapping pairs."""
import numpy as np
import pytest

from stream_b200 import workloads

pytestmark = pytest.mark.gpu

TOPO = ("child_left", "child_right", "parent", "bboxes", "subtree_size", "sah", "obj_m", "root")


def _same(a, b):
    a, b = np.atleast_1d(np.asarray(a)), np.atleast_1d(np.asarray(b))
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def _xyzr(pts, r):
    return np.concatenate([pts, np.broadcast_to(np.float32(r), (len(pts), 1))], axis=1).astype(np.float32)


def _gpu(xyzr, K=7, area3d=True, rounds=3):
    from stream_b200.geometry import Sphere3DTRBVH
    t = Sphere3DTRBVH()
    t.set_objects(xyzr, treelet_size=K, area3d=area3d, rounds=rounds)
    assert t.build() == 0
    return t


@pytest.mark.parametrize("n", [2, 3, 64, 5000])
def test_apetrei_matches_reference_build(sb, reference, n):
    rng = np.random.default_rng(n)
    xyzr = np.concatenate([rng.random((n, 3)), 0.01 * (1 + rng.random((n, 1)))], 1).astype(np.float32)
    got = _gpu(xyzr, K=5, area3d=False, rounds=0).arrays()
    want = reference.trbvh3d(xyzr, optimize=False)
    for k in ("child_left", "child_right", "range_min", "range_max", "parent", "bboxes", "subtree_size", "obj_m",
              "root"):
        assert _same(got[k], want[k]), k


@pytest.mark.parametrize("K,area3d", [(5, False), (7, True), (8, True)])
@pytest.mark.parametrize("n", [100, 20_000])
def test_restructured_tree_matches_oracle(sb, restate, K, area3d, n):
    pts, _ = workloads.uniform_cube(n, seed=K + n)
    xyzr = _xyzr(pts, 0.3 * n ** (-1 / 3))
    got = _gpu(xyzr, K=K, area3d=area3d).arrays()
    want = restate.trbvh3d(xyzr, treelet_size=K, area3d=area3d, rounds=3)
    for k in TOPO:
        assert _same(got[k], want[k]), k


@pytest.mark.parametrize("n,seed", [(64, 1), (2000, 8), (20_000, 3)])
def test_restructured_tree_matches_reference_build(sb, reference, n, seed):
    """The reference's full build (Apetrei + three rounds of 5-leaf treelet
    restructuring with its 2D SAH area, include/geometry/trbvh.hpp:637-679) on
    spheres of radius 0, where its arrival-order SAH sums are deterministic
    with one OpenMP thread: the GPU tree equals it bit for bit."""
    rng = np.random.default_rng(seed)
    xyzr = np.concatenate([rng.random((n, 3)), np.zeros((n, 1))], 1).astype(np.float32)
    got = _gpu(xyzr, K=5, area3d=False, rounds=3).arrays()
    want = reference.trbvh3d(xyzr, optimize=True, threads=1)
    for k in TOPO + ("range_min", "range_max"):
        assert _same(got[k], want[k]), k


@pytest.mark.parametrize("n", [2, 3, 5000, 100_003])
def test_lbvha_matches_reference_build(sb, reference, n):
    """Sphere3DLBVHa (the Apetrei build) against the reference's LBVHa
    (include/geometry/lbvh_agglo.hpp): children, ranges, parents, boxes, root
    and sorted objects bit for bit."""
    from stream_b200.geometry import Sphere3DLBVHa
    rng = np.random.default_rng(n + 7)
    xyzr = np.concatenate([rng.random((n, 3)), 0.01 * (1 + rng.random((n, 1)))], 1).astype(np.float32)
    t = Sphere3DLBVHa()
    t.set_objects(xyzr)
    assert t.build() == 0
    got, want = t.arrays(), reference.lbvha3d(xyzr)
    for k in ("children", "range", "parent", "bboxes", "root", "obj_m"):
        assert _same(got[k], want[k]), k


def test_restructuring_lowers_sah(sb):
    pts, a = workloads.meshing_stress(100_000, seed=2)
    xyzr = _xyzr(pts, a[0])
    before = _gpu(xyzr, rounds=0).arrays()
    after = _gpu(xyzr, rounds=3).arrays()
    assert after["sah"][after["root"]] <= before["sah"][before["root"]]


def test_overlap_queries(sb, restate):
    rng = np.random.default_rng(1)
    n = 3000
    xyzr = np.concatenate([rng.random((n, 3)), 0.25 * n ** (-1 / 3) * (1 + rng.random((n, 1)))], 1).astype(np.float32)
    t = _gpu(xyzr)
    got = t.count_overlaps()
    o = t.arrays()["obj_m"]
    d2 = ((o[:, None, :3] - o[None, :, :3]) ** 2).sum(-1)
    rs = (o[:, None, 3] + o[None, :, 3]) ** 2
    brute = (d2 <= rs).sum(1) - 1
    assert np.array_equal(got, brute)
    assert np.array_equal(got, restate.trbvh3d(xyzr, count=True)["count"])


@pytest.mark.slow
def test_meshing_stress_4m_treelet7(sb):
    """Full-size meshing-stress cloud, treelet size 7: a valid tree (every
    node's box holds its children's, subtree sizes add up) with lower SAH."""
    pts, a = workloads.meshing_stress(4_000_000, seed=0)
    xyzr = _xyzr(pts, a[0])
    t = _gpu(xyzr, K=7)
    g = t.arrays()
    n = len(pts)
    cl, cr = g["child_left"].astype(np.int64), g["child_right"].astype(np.int64)
    ids = np.arange(n, 2 * n - 1)
    sz = g["subtree_size"]
    assert np.array_equal(sz[ids], sz[cl] + sz[cr])
    assert sz[g["root"]] == n
    b = g["bboxes"]
    for c in (cl, cr):
        assert np.all(b[ids, :3] <= b[c, :3]) and np.all(b[ids, 3:] >= b[c, 3:])
    kids = np.concatenate([cl, cr])
    assert np.array_equal(np.sort(kids), np.delete(np.arange(2 * n - 1), g["root"]))
