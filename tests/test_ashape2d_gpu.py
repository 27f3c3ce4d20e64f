"""2D alpha shape on the GPU vs the oracle (src/mesh/DirectAlphaShape2D.cpp):
bit-exact permutation, neighbour lists, triangles, CSR edges, boundary-edge and
boundary-node flags on seeded clouds, the reference's golden fixtures,
degenerate inputs (co-circular lattice, duplicates, collinear points, tiny
coordinates, the 250-id fill limit) and the published 1M-point triangle count."""
import glob
import os

import numpy as np
import pytest

from stream_b200 import workloads

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _run(pts, alpha):
    from stream_b200.mesh import AlphaShape2D
    a = AlphaShape2D()
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
    assert np.array_equal(got["nodes"], want.coords_m[:n, :2]), tag + " ordered nodes"
    assert np.array_equal(got["nineig"], want.nineig), tag + " star sizes"
    w = min(got["cand"].shape[1], want.cand.shape[1])
    valid = np.arange(w)[None, :] < (want.nineig[:, None].astype(np.int64) - 3)
    assert np.array_equal(np.where(valid, got["cand"][:, :w], 0), np.where(valid, want.cand[:, :w], 0)), \
        tag + " neighbours"
    assert np.array_equal(got["nelem"], want.nelem), tag + " kept triangles per star"
    assert np.array_equal(got["node_is_bnd"], want.node_is_bnd), tag + " boundary nodes"
    assert np.array_equal(got["row"], want.row), tag + " edge rows"
    assert np.array_equal(got["neig"], want.neig), tag + " edges"
    assert np.array_equal(got["edge_is_bnd"], want.edge_is_bnd), tag + " boundary edges"
    assert got["elems"].shape == want.elems.shape, tag + " triangle count"
    assert np.array_equal(got["elems"], want.elems), tag + " triangles"


@pytest.mark.parametrize("n,seed", [(20, 0), (1000, 1), (50_000, 2)])
def test_uniform(sb, restate, n, seed):
    pts, al = workloads.uniform_square(n, seed)
    _compare(_run(pts, al), restate.ashape2d(pts, al), f"uniform {n}")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ashape2d_*.npz"))),
                         ids=lambda p: os.path.basename(p))
def test_reference_golden(sb, path):
    g = np.load(path)
    got = _run(g["pts"], g["alpha"])
    for k in ("perm", "elems", "row", "neig", "edge_is_bnd", "node_is_bnd", "nineig", "nelem"):
        assert np.array_equal(got[k], g[k]), k


def test_lattice_cocircular(sb, restate):
    """40 x 40 lattice: every unit square is co-circular, so the exact stage and
    Simulation of Simplicity decide the triangulation."""
    pts, al = workloads.lattice2d(40)
    got = _run(pts, al)
    want = restate.ashape2d(pts, al)
    assert want.n_exact > 0 and got["counters"]["exact_calls"] > 0
    _compare(got, want, "lattice")


def test_fill_limit(sb, restate):
    """alpha 0.2 on a 40 x 40 lattice: stars stop filling at 250 local ids as
    in the reference (DirectAlphaShape2D.cpp:351-354)."""
    pts, al = workloads.lattice2d(40, alpha=0.2)
    got = _run(pts, al)
    want = restate.ashape2d(pts, al)
    assert got["counters"]["fill_limited"] > 0
    _compare(got, want, "fill limit")


def test_degenerate_inputs(sb, restate):
    rng = np.random.default_rng(3)
    u = rng.random((3000, 2)).astype(np.float32)
    circ = np.stack([np.cos(np.arange(300) * (2 * np.pi / 300)), np.sin(np.arange(300) * (2 * np.pi / 300))], 1)
    cases = {
        "duplicates": (np.concatenate([u, u[:400]]), np.full(3400, 0.04, np.float32)),
        "cocircular": (np.concatenate([circ, [[0.0, 0.0]]]).astype(np.float32), np.full(301, 0.5, np.float32)),
        "collinear": (np.stack([np.linspace(0, 1, 200), np.zeros(200)], 1).astype(np.float32),
                      np.full(200, 0.02, np.float32)),
        "tiny_coords": ((rng.random((1500, 2)) * 1e-6).astype(np.float32), np.full(1500, 1e-7, np.float32)),
        "variable_alpha": (u, (rng.random(3000) * 0.05 + 0.005).astype(np.float32)),
        "two_points": (np.array([[0, 0], [0.01, 0]], np.float32), np.full(2, 0.1, np.float32)),
    }
    for name, (pts, al) in cases.items():
        _compare(_run(pts, al), restate.ashape2d(pts, al), name)


def test_dambreak_column(sb, restate):
    pts, al = workloads.dambreak_column2d(h=0.004, seed=1)
    _compare(_run(pts, al), restate.ashape2d(pts, al), "column")


def test_published_1m_case(sb, restate):
    """uniform2D -n 1000000 -a 0.0012 (testcases/IMR26/README.md:48-54):
    1,877,465 triangles, and every output equal to the oracle's."""
    pts, al = workloads.glibc_uniform_square(1_000_000, 0.0012)
    got = _run(pts, al)
    assert len(got["elems"]) == 1_877_465
    _compare(got, restate.ashape2d(pts, al), "uniform2D 1M")


def test_reuse_handle(sb, restate):
    """One handle, two clouds of different sizes: buffers are resized."""
    from stream_b200.mesh import AlphaShape2D
    a = AlphaShape2D()
    for n, seed in [(5000, 4), (800, 5)]:
        pts, al = workloads.uniform_square(n, seed)
        a.set_nodes(pts, al)
        a.compute()
        assert np.array_equal(a.get_elem(), restate.ashape2d(pts, al).elems)


@pytest.mark.parametrize("dim", [2, 3])
def test_mesh_point_cloud_file(sb, restate, tmp_path, dim):
    """.bin point cloud in, elems.txt / nodes.txt out, as the reference's
    run_on_simulation_meshes.py and uniform harnesses use them."""
    from stream_b200 import io as sio
    if dim == 2:
        pts, al = workloads.dambreak_column2d(h=0.01, seed=3)
        want = restate.ashape2d(pts, al)
    else:
        pts, al = workloads.dambreak_column(h=0.05, seed=3)
        want = restate.ashape3d(pts, al)
    sio.write_point_cloud(tmp_path / "cloud.bin", pts, al)
    elems, nodes = sio.mesh_point_cloud(tmp_path / "cloud.bin", dim, out_dir=tmp_path)
    assert np.array_equal(elems, want.elems)
    assert np.array_equal(sio.read_elems_txt(tmp_path / "elems.txt", dim), want.elems)
    assert np.allclose(sio.read_nodes_txt(tmp_path / "nodes.txt", dim), want.coords_m[:len(pts), :dim], atol=6e-6)


def test_device_input_stream_and_profile(sb, restate):
    """Additive 2D API: points already on the GPU (float4 x, y, 0, alpha), a
    caller-owned stream, and the per-stage profile."""
    import ctypes
    import torch
    from stream_b200 import libmesh
    from stream_b200.mesh import AlphaShape2D
    pts, al = workloads.uniform_square(20_000, seed=6)
    x = torch.zeros((len(pts), 4), dtype=torch.float32, device="cuda")
    x[:, :2] = torch.from_numpy(pts).cuda()
    x[:, 3] = torch.from_numpy(al).cuda()
    s = torch.cuda.Stream()
    a = AlphaShape2D()
    libmesh.AlphaShape2D_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    assert libmesh.AlphaShape2D_set_stream(a.mesh, ctypes.c_void_p(s.cuda_stream)) == 0
    a.set_profiling(True)
    assert libmesh.AlphaShape2D_set_nodes_device(a.mesh, len(pts), ctypes.c_void_p(x.data_ptr())) == 0
    a.nnodes = len(pts)
    a.init()
    a.compute()
    want = restate.ashape2d(pts, al)
    assert np.array_equal(a.get_elem(), want.elems)
    assert np.array_equal(a.get_permutation(), want.perm)
    prof = a.profile()
    assert set(prof) == {"lbvh", "count_pass", "fill_pass", "star", "scan", "compress"}
    assert all(v >= 0.0 for v in prof.values()) and prof["star"] > 0.0
    assert libmesh.AlphaShape2D_set_stream(a.mesh, None) == 0
