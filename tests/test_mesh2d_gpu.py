"""GPU: the 2D Delaunay mesher behind the reference's Mesh2D interface
(src/mesh/mesh.cpp:806-862).

The reference's own insertion phases overrun a fixed-size traversal heap
(mesh.cpp:471, 509, 548), so its output is not an oracle.  Pinned to the
reference: the Morton order and the super nodes of Mesh2D_init (fixtures
from its build, tests/golden/make_golden.py).  Oracle for the triangles:
Qhull (scipy.spatial.Delaunay, FP64) on the ordered points plus the super
nodes, the super triangles left out -- on inputs in general position, where
the triangulation is unique.  Qhull decides in floating point: where the
two differ (a near co-circular quadrilateral split the other way), exact
rational arithmetic must show the mesher's triangles empty-circled and
Qhull's not, over the same area.  On a lattice (every square co-circular) the
output is checked for being a Delaunay triangulation of the unit square:
positive orientation, total area 1, every interior edge shared by two
triangles, and no point strictly inside any circumcircle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PHASES = {"morton": "insert_morton_neighbors", "bvh": "insert_BVH_neighbors", "iterative": "insert_iterative"}


def _mesh(xy, phases=("morton", "bvh", "iterative"), drop=True):
    from stream_b200.mesh import Mesh2D
    m = Mesh2D()
    m.set_nodes(xy)
    for ph in phases:
        getattr(m, PHASES[ph])()
    if drop:
        m.remove_super_nodes()
    return m, m.get_elem()


def _tri_set(e):
    return {tuple(sorted(map(int, t))) for t in e}


def _qhull(points):
    from scipy.spatial import Delaunay
    return _tri_set(Delaunay(points.astype(np.float64)).simplices)


def _orient(xo, e):
    a, b, c = (xo[e[:, k]].astype(np.float64) for k in range(3))
    return (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])


def _exact_disagreement_ok(xo, ours, theirs):
    """The triangles only one side has: few, covering the same area, and the
    mesher's have no vertex of the other set strictly inside their circles
    (exact rationals on the float32 coordinates), while each of Qhull's has one."""
    from fractions import Fraction
    if not ours and not theirs:
        return True
    if len(ours) != len(theirs) or len(ours) > 16:
        return False
    pts = {i: (Fraction(float(xo[i, 0])), Fraction(float(xo[i, 1]))) for t in ours | theirs for i in t}

    def orient(a, b, c):
        return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])

    def inside(t, d):
        a, b, c = (pts[i] for i in t)
        if orient(a, b, c) < 0:
            b, c = c, b
        rows = [(p[0] - d[0], p[1] - d[1]) for p in (a, b, c)]
        lift = [x * x + y * y for x, y in rows]
        (ax, ay), (bx, by), (cx, cy) = rows
        return ax * (by * lift[2] - lift[1] * cy) - ay * (bx * lift[2] - lift[1] * cx) + lift[0] * (bx * cy - by * cx)

    def area(ts):
        return sum(abs(orient(*(pts[i] for i in t))) for t in ts)

    verts = set(pts)
    mine_ok = all(inside(t, pts[v]) <= 0 for t in ours for v in verts - set(t))
    theirs_bad = all(any(inside(t, pts[v]) >= 0 for v in verts - set(t)) for t in theirs)
    return mine_ok and theirs_bad and area(ours) == area(theirs)


def _check_against_qhull(xy, **kw):
    m, e = _mesh(xy, **kw)
    n = len(xy)
    assert m.status == 0, m.status
    assert m.counters()["incomplete"] == 0
    xo = m.get_ordered_nodes()
    assert np.array_equal(xo, xy[m.get_permutation()])
    sup = m.get_super_nodes()
    full = _qhull(np.concatenate([xo, sup]))
    want = {t for t in full if t[2] < n}
    got = _tri_set(e)
    assert len(got) == len(e), "a triangle written twice"
    assert _exact_disagreement_ok(xo, got - want, want - got), (len(got), len(want), got - want, want - got)
    assert np.all(e[:, 0] < e[:, 1]) and np.all(e[:, 0] < e[:, 2]), "owner (smallest id) first"
    assert np.all(_orient(xo, e) > 0), "counter-clockwise"
    return m, e, full


@pytest.mark.parametrize("name", ["mesh2d_uniform_3000", "mesh2d_blobs_2000", "mesh2d_lattice_30"])
def test_order_and_super_nodes_match_reference(name):
    import os
    from stream_b200.mesh import Mesh2D
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", name + ".npz"))
    m = Mesh2D()
    m.set_nodes(g["xy"])
    assert np.array_equal(m.get_permutation(), g["perm"])
    assert np.array_equal(m.get_super_nodes(), g["super_nodes"])
    assert np.array_equal(m.get_ordered_nodes(), g["xy"][g["perm"]])


@pytest.mark.parametrize("n,seed", [(3000, 1), (50_000, 2), (200_000, 3)])
def test_uniform_matches_qhull(n, seed):
    xy = np.random.default_rng(seed).random((n, 2)).astype(np.float32)
    _check_against_qhull(xy)


def test_clustered_matches_qhull():
    rng = np.random.default_rng(4)
    c = rng.random((16, 2))
    xy = (c[rng.integers(0, 16, 60_000)] + 0.004 * rng.standard_normal((60_000, 2))).astype(np.float32)
    xy = np.unique(xy, axis=0)
    _check_against_qhull(rng.permutation(xy))


def test_anisotropic_strip_matches_qhull():
    rng = np.random.default_rng(5)
    xy = np.stack([rng.random(20_000) * 100.0, rng.random(20_000) * 0.01], 1).astype(np.float32)
    _check_against_qhull(xy)


@pytest.mark.parametrize("phases", [("iterative",), ("morton", "iterative"), ("bvh", "iterative"),
                                    ("morton", "bvh", "bvh", "iterative")])
def test_phase_orders_give_the_same_triangulation(phases):
    xy = np.random.default_rng(6).random((20_000, 2)).astype(np.float32)
    _check_against_qhull(xy, phases=phases)


def test_super_triangles_kept_without_remove_super_nodes():
    xy = np.random.default_rng(7).random((5000, 2)).astype(np.float32)
    m, e = _mesh(xy, drop=False)
    xo = m.get_ordered_nodes()
    full = _qhull(np.concatenate([xo, m.get_super_nodes()]))
    got = _tri_set(e)
    assert _exact_disagreement_ok(np.concatenate([xo, m.get_super_nodes()]), got - full, full - got)
    assert e.max() >= len(xy)  # super nodes are ids n..n+2


@pytest.mark.parametrize("n", [2, 3, 5, 17])
def test_tiny_inputs(n):
    xy = np.random.default_rng(100 + n).random((n, 2)).astype(np.float32)
    _check_against_qhull(xy)


def test_collinear_points_have_no_inner_triangle():
    xy = np.stack([np.linspace(0, 1, 50), np.linspace(0, 1, 50)], 1).astype(np.float32)
    m, e = _mesh(xy)
    assert len(e) == 0
    assert m.counters()["incomplete"] == 0


def _incircle(a, b, c, d):
    """> 0 when d is inside the circle of the counter-clockwise a, b, c (FP64)."""
    m = np.stack([a - d, b - d, c - d], 1)
    lift = (m ** 2).sum(-1)
    return (m[:, 0, 0] * (m[:, 1, 1] * lift[:, 2] - lift[:, 1] * m[:, 2, 1])
            - m[:, 0, 1] * (m[:, 1, 0] * lift[:, 2] - lift[:, 1] * m[:, 2, 0])
            + lift[:, 0] * (m[:, 1, 0] * m[:, 2, 1] - m[:, 1, 1] * m[:, 2, 0]))


@pytest.mark.parametrize("k", [2, 3, 12, 30])
def test_lattice_is_a_delaunay_triangulation(k):
    g = np.arange(k, dtype=np.float32) / (k - 1)
    xy = np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)
    m, e = _mesh(xy)
    assert m.counters()["incomplete"] == 0 and m.status == 0
    xo = m.get_ordered_nodes().astype(np.float64)
    o = _orient(xo, e)
    assert np.all(o > 0)
    assert abs(o.sum() / 2 - 1.0) < 1e-9, o.sum() / 2  # the unit square exactly covered
    assert len(e) == 2 * (k - 1) ** 2
    edges = {}
    for t in e:
        for u, v in ((t[0], t[1]), (t[1], t[2]), (t[2], t[0])):
            key = (min(u, v), max(u, v))
            edges[key] = edges.get(key, 0) + 1
    assert max(edges.values()) <= 2
    assert sum(1 for c in edges.values() if c == 1) == 4 * (k - 1)  # the square's boundary
    a, b, c = xo[e[:, 0]], xo[e[:, 1]], xo[e[:, 2]]
    for d in xo:
        assert np.all(_incircle(a, b, c, np.broadcast_to(d, a.shape)) < 1e-12)


def test_bad_input_rejected():
    from stream_b200 import StreamError
    from stream_b200.mesh import Mesh2D
    m = Mesh2D()
    with pytest.raises(StreamError):
        m.set_nodes(np.array([[0.0, 0.0], [np.nan, 1.0], [1.0, 1.0]], np.float32))
    with pytest.raises(StreamError):
        m.set_nodes(np.zeros((1, 2), np.float32))


def test_duplicate_points_end_with_a_bounded_run():
    """Coincident points have no Delaunay triangulation: every phase still
    ends (each star's queries and local ids are bounded) and the distinct
    points' triangles away from the duplicates stay Delaunay."""
    rng = np.random.default_rng(8)
    xy = rng.random((2000, 2)).astype(np.float32)
    xy = np.concatenate([xy, xy[:20]])
    m, e = _mesh(xy)
    assert not m.status & 0x180  # no bad input, no CUDA error
    assert len(e) > 3000


def test_many_coincident_points_stay_bounded():
    """50 sites with 40 copies each among 15,000 distinct points.  The copies
    have no triangulation; their equal Morton codes deepen the LBVH past the
    traversal stack (reported, and raised by the Python class) and their
    stars meet circles that cannot be bounded, whose queries give up after a
    fixed number of points or LBVH nodes.  What is checked: every phase ends
    quickly, with no CUDA error, bad input or exact-stage overflow."""
    import time
    from stream_b200 import StreamError
    from stream_b200.mesh import Mesh2D
    rng = np.random.default_rng(9)
    sites = np.repeat(rng.random((50, 2)), 40, axis=0)
    xy = rng.permutation(np.concatenate([rng.random((15_000, 2)), sites])).astype(np.float32)
    m = Mesh2D()
    m.set_nodes(xy)
    t0 = time.perf_counter()
    for ph in PHASES.values():
        try:
            getattr(m, ph)()
        except StreamError:
            pass
    assert time.perf_counter() - t0 < 60.0
    assert not m.status & 0x190, m.status
