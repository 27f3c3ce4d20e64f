"""Regenerate the golden fixtures of this directory from the reference itself.

Runs the reference's own sources (oracle/_ref/libstream_ref.so: the
unmodified src/mesh/DirectAlphaShape3D.cpp, src/mesh/DirectAlphaShape2D.cpp,
include/geometry/lbvh.hpp, lbvh_agglo.hpp, trbvh.hpp and src/numerics/*.cpp
built for the host against oracle/ava_shim) on small seeded inputs and stores inputs and outputs as compressed .npz files.  Needs the
reference build (`make -C oracle ref`, which needs the reference tree).

Usage: python tests/golden/make_golden.py [mesh2d]   (all fixtures, or only the Mesh2D ones)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Reference  # noqa: E402
from stream_b200 import workloads  # noqa: E402  (pure-Python generators)


def cases():
    yield "ashape_uniform_3000", *workloads.uniform_cube(3000, seed=42)
    yield "ashape_lattice_9", *workloads.lattice(9)
    pts, al = workloads.meshing_stress(6000, seed=9)
    yield "ashape_stress_6000", pts, al
    pts, al = workloads.dambreak_column(h=0.05, seed=2)
    yield "ashape_column", pts, al


def cases2d():
    yield "ashape2d_uniform_4000", *workloads.uniform_square(4000, seed=42)
    yield "ashape2d_lattice_40", *workloads.lattice2d(40)
    yield "ashape2d_column", *workloads.dambreak_column2d(h=0.02, seed=2)
    yield "ashape2d_glibc_10000", *workloads.glibc_uniform_square(10000, 0.024)


def cases_mesh2d():
    rng = np.random.default_rng(11)
    yield "mesh2d_uniform_3000", rng.random((3000, 2)).astype(np.float32)
    c = rng.random((8, 2))
    yield "mesh2d_blobs_2000", (c[rng.integers(0, 8, 2000)] + 0.01 * rng.standard_normal((2000, 2))).astype(np.float32)
    g = np.arange(30, dtype=np.float32) / 29
    yield "mesh2d_lattice_30", np.stack(np.meshgrid(g, g, indexing="ij"), -1).reshape(-1, 2)


def mesh2d(ref):
    """Morton order and super nodes of the reference's Mesh2D_init (its
    insertion phases overrun a fixed-size heap and are not run)."""
    for name, xy in cases_mesh2d():
        perm, coords_m = ref.mesh2d_order(xy)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), xy=xy, perm=perm, super_nodes=coords_m[len(xy):])
        print(name, len(xy), "points")


def main(parts):
    ref = Reference()
    if parts == ["mesh2d"]:
        mesh2d(ref)
        return
    mesh2d(ref)
    for name, pts, al in cases2d():
        r = ref.ashape2d(pts, al)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), pts=pts, alpha=al, perm=r.perm, elems=r.elems,
                            row=r.row, neig=r.neig, edge_is_bnd=r.edge_is_bnd, node_is_bnd=r.node_is_bnd,
                            nineig=r.nineig, nelem=r.nelem)
        print(name, len(pts), "points", len(r.elems), "triangles")
    for name, pts, al in cases():
        r = ref.ashape3d(pts, al)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), pts=pts, alpha=al, perm=r.perm, elems=r.elems,
                            row=r.row, neig=r.neig, edge_is_bnd=r.edge_is_bnd, node_is_bnd=r.node_is_bnd,
                            nineig=r.nineig)
        print(name, len(pts), "points", len(r.elems), "tets")
    pts, _ = workloads.uniform_cube(1500, seed=5)
    xyzr = np.concatenate([pts, np.full((len(pts), 1), 0.02, np.float32)], 1)
    g = ref.lbvh3d(xyzr)
    np.savez_compressed(os.path.join(HERE, "lbvh_uniform_1500.npz"), xyzr=xyzr, **g)
    print("lbvh_uniform_1500")
    # LBVHa, Apetrei's agglomerative build (include/geometry/lbvh_agglo.hpp)
    pts, _ = workloads.uniform_cube(1500, seed=6)
    xyzr = np.concatenate([pts, np.full((len(pts), 1), 0.02, np.float32)], 1)
    np.savez_compressed(os.path.join(HERE, "lbvha_uniform_1500.npz"), xyzr=xyzr, **ref.lbvha3d(xyzr))
    print("lbvha_uniform_1500")
    # TRBVH with treelet restructuring (include/geometry/trbvh.hpp:637-679) on
    # spheres of radius 0, one thread: deterministic SAH sums
    xyzr = np.concatenate([workloads.uniform_cube(2000, seed=8)[0], np.zeros((2000, 1), np.float32)], 1)
    t = ref.trbvh3d(xyzr, optimize=True, threads=1)
    np.savez_compressed(os.path.join(HERE, "trbvh_r0_2000.npz"), xyzr=xyzr, **t)
    print("trbvh_r0_2000")


if __name__ == "__main__":
    main(sys.argv[1:])
