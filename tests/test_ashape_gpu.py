"""3D alpha shape on the GPU vs the oracle (src/mesh/DirectAlphaShape3D.cpp):
bit-exact permutation, candidate lists, tets, CSR edges, boundary-edge and
free-surface flags on seeded clouds, degenerate lattices and truncated stars."""
import numpy as np
import pytest

from stream_b200 import workloads

pytestmark = pytest.mark.gpu


def _run(pts, alpha, bits=63):
    from stream_b200.mesh import AlphaShape3D
    a = AlphaShape3D(morton_bits=bits)
    a.set_nodes(pts, alpha)
    a.compute()
    row, neig, ebnd = a.get_edges()
    nineig, nkeep, cand = a.get_stars()
    return dict(elems=a.get_elem(), perm=a.get_permutation(), row=row, neig=neig, edge_is_bnd=ebnd,
                node_is_bnd=a.get_boundary_nodes(), nineig=nineig, nelem=nkeep, cand=cand,
                nodes=a.get_ordered_nodes(), counters=a.counters())


def _compare(got, want, tag=""):
    n = len(want.perm)
    assert np.array_equal(got["perm"], want.perm), tag + " perm"
    assert np.array_equal(got["nodes"], want.coords_m[:n, :3]), tag + " ordered nodes"
    assert np.array_equal(got["nineig"], want.nineig), tag + " star sizes"
    valid = np.arange(124)[None, :] < (want.nineig[:, None].astype(np.int64) - 4)
    assert np.array_equal(np.where(valid, got["cand"], 0), np.where(valid, want.cand, 0)), tag + " candidates"
    assert np.array_equal(got["nelem"], want.nelem), tag + " kept tets per star"
    assert np.array_equal(got["node_is_bnd"], want.node_is_bnd), tag + " free-surface flags"
    assert np.array_equal(got["row"], want.row), tag + " edge rows"
    assert np.array_equal(got["neig"], want.neig), tag + " edges"
    assert np.array_equal(got["edge_is_bnd"], want.edge_is_bnd), tag + " boundary edges"
    assert got["elems"].shape == want.elems.shape, tag + " tet count"
    assert np.array_equal(got["elems"], want.elems), tag + " tets"


@pytest.mark.parametrize("n,seed", [(50, 0), (1000, 1), (20_000, 2)])
def test_uniform(sb, restate, n, seed):
    pts, al = workloads.uniform_cube(n, seed)
    got = _run(pts, al)
    _compare(got, restate.ashape3d(pts, al), f"uniform {n}")


def test_uniform_30bit(sb, restate):
    pts, al = workloads.uniform_cube(5000, 7)
    got = _run(pts, al, bits=30)
    _compare(got, restate.ashape3d(pts, al, bits=30), "uniform 30-bit")


def test_lattice_degenerate(sb, restate):
    """12^3 lattice: nearly every insphere test is exactly co-spherical, so the
    exact stage and Simulation of Simplicity decide the connectivity."""
    pts, al = workloads.lattice(12)
    got = _run(pts, al)
    want = restate.ashape3d(pts, al)
    assert want.n_exact > 0 and got["counters"]["exact_calls"] > 0
    _compare(got, want, "lattice")


def test_lattice_near_origin(sb, restate):
    """Lattice sites k/99 near the origin: FP32 expansion tails can underflow in
    the reference's exact path; the GPU must repeat its float sequence."""
    g = np.stack(np.meshgrid(*[np.arange(10)] * 3, indexing="ij"), -1).reshape(-1, 3) / 99.0
    pts = g.astype(np.float32)
    al = np.full(len(pts), 1.5 / 99.0, np.float32)
    _compare(_run(pts, al), restate.ashape3d(pts, al), "lattice near origin")


def test_meshing_stress_small(sb, restate):
    """Scaled-down meshing-stress mix (uniform + blobs + lattice): truncated
    stars, degeneracies and variable density together."""
    pts, al = workloads.meshing_stress(30_000, seed=5)
    got = _run(pts, al)
    want = restate.ashape3d(pts, al)
    assert want.n_truncated > 0
    _compare(got, want, "meshing stress")


def test_variable_alpha_and_duplicates(sb, restate):
    rng = np.random.default_rng(11)
    pts = rng.random((3000, 3)).astype(np.float32)
    pts = np.concatenate([pts, pts[:50]])
    al = (0.03 + 0.05 * rng.random(len(pts))).astype(np.float32)
    got = _run(pts, al)
    want = restate.ashape3d(pts, al)
    # Coincident points make the reference read outside its cavity-cycle table
    # (undefined behaviour); both sides stop that star and flag it.
    assert (want.status & 4) and (got["counters"]["status"] & 4)
    _compare(got, want, "variable alpha + duplicates")


def test_tiny_inputs(sb, restate):
    for n in (2, 3, 4, 5, 8):
        pts, al = workloads.uniform_cube(n, seed=n)
        al[:] = 2.0
        _compare(_run(pts, al), restate.ashape3d(pts, al), f"tiny {n}")


def test_dambreak_column(sb, restate):
    pts, al = workloads.dambreak_column(h=0.04, seed=1)
    _compare(_run(pts, al), restate.ashape3d(pts, al), "dam-break column")


@pytest.mark.slow
def test_config1_200k(sb, restate):
    """Plain-method case: 200,000 uniform points, alpha = 1.3 N^-1/3."""
    pts, al = workloads.uniform_cube(200_000, seed=0)
    _compare(_run(pts, al), restate.ashape3d(pts, al), "200k")


def test_conflict_predicate_batch(sb, restate):
    """The three-stage conflict decision vs the reference decision on hard
    quintuples: co-spherical lattice points, tiny coordinates (underflow of
    FP32 expansion tails), near-degenerate perturbations and random ones."""
    from stream_b200 import lib
    import ctypes
    rng = np.random.default_rng(0)
    cases = []
    # cospherical: 5 vertices of a unit cube scaled near the origin and far
    cube = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1]], float)
    for s in (1 / 99.0, 3 / 99.0, 1e-3, 0.37, 1.0):
        for o in (0.0, 1 / 99.0, 0.5):
            for _ in range(40):
                sel = rng.choice(8, 5, replace=False)
                cases.append((cube[sel] * s + o))
    # near-degenerate: cospherical + 1-ulp perturbations
    for _ in range(2000):
        sel = rng.choice(8, 5, replace=False)
        p = (cube[sel] * rng.choice([0.01, 0.1, 1 / 99.0]) + rng.random(3) * 0.1).astype(np.float32)
        k = rng.integers(0, 5)
        p[k] = np.nextafter(p[k], np.float32(1.0))
        cases.append(p.astype(float))
    for _ in range(3000):
        cases.append(rng.random((5, 3)) * rng.choice([1.0, 1e-3, 1e-5]))
    # the FP64 stage's range [2^-60, 2^20) below 2^-6, where the reference's
    # FP32 expansions can underflow: random and 1-ulp-perturbed co-spherical
    # quintuples at tiny scales, and tiny points next to moderate ones
    for sc in (2.0 ** -8, 2.0 ** -12, 2.0 ** -20, 2.0 ** -30, 2.0 ** -40, 2.0 ** -55):
        for _ in range(300):
            cases.append(rng.random((5, 3)) * sc)
        for _ in range(300):
            sel = rng.choice(8, 5, replace=False)
            p = (cube[sel] * sc * rng.choice([1.0, 3.0, 0.37]) + rng.random(3) * sc).astype(np.float32)
            k = rng.integers(0, 5)
            p[k] = np.nextafter(p[k], np.float32(1.0))
            cases.append(p.astype(float))
        for _ in range(100):
            q = rng.random((5, 3)) * sc
            q[rng.integers(0, 5)] += 0.3
            cases.append(q)
    pts = np.array(cases, dtype=np.float32)
    ids = np.stack([rng.permutation(1000)[:5] for _ in range(len(pts))]).astype(np.uint32)
    want, used = restate.conflict_batch(pts, ids)
    got = np.zeros(len(pts), np.float32)
    P = ctypes.c_void_p
    lib.stream_b200_conflict_batch.argtypes = [ctypes.c_uint32, P, P, P]
    rc = lib.stream_b200_conflict_batch(len(pts), pts.ctypes.data_as(P), ids.ctypes.data_as(P), got.ctypes.data_as(P))
    assert rc == 0
    assert used.sum() > 100
    assert np.array_equal(np.sign(got) > 0, np.sign(want) > 0)


def test_work_counting_build_same_outputs(sb, restate):
    """The counting build of the star pass (profiling runs) decides exactly as
    the timed one and reports its stage-1 / stage-2 work."""
    import ctypes
    from stream_b200 import libmesh
    from stream_b200.mesh import AlphaShape3D
    pts, al = workloads.meshing_stress(20_000, seed=4)
    plain = _run(pts, al)
    a = AlphaShape3D()
    libmesh.AlphaShape3D_set_work_counters.argtypes = [ctypes.c_void_p, ctypes.c_int]
    libmesh.AlphaShape3D_get_work.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    assert libmesh.AlphaShape3D_set_work_counters(a.mesh, 1) == 0
    a.set_nodes(pts, al)
    a.compute()
    work = np.zeros(2, np.uint64)
    assert libmesh.AlphaShape3D_get_work(a.mesh, work.ctypes.data_as(ctypes.c_void_p)) == 0
    assert np.array_equal(a.get_elem(), plain["elems"])
    assert work[0] > 0 and work[1] <= work[0]
