"""File formats of the reference's mesher test cases.

* Point clouds (``testcases/IMR26/README.md:137-145``,
  ``run_on_simulation_meshes.py:82,128``): a flat little-endian float32 array
  of records (x, y, alpha) in 2D or (x, y, z, alpha) in 3D, no header.
* Mesh dumps of the uniform2D / uniform3D harnesses
  (``testcases/IMR26/uniform2D.cpp:183-201``, ``uniform3D.cpp:183-201``):
  ``elems.txt`` holds one element per line as ``"%u %u %u"`` (2D) or
  ``"%u %u %u %u"`` (3D) in Morton-ordered ids, and ``nodes.txt`` the
  Morton-ordered coordinates as ``"%.5f %.5f"`` / ``"%.5f %.5f %.5f"``.
"""
from __future__ import annotations

import os

import numpy as np


def read_point_cloud(path: str | os.PathLike, dim: int) -> tuple[np.ndarray, np.ndarray]:
    """(coords (N, dim) float32, alpha (N,) float32) from a .bin point cloud."""
    if dim not in (2, 3):
        raise ValueError("dim must be 2 or 3")
    raw = np.fromfile(path, dtype="<f4")
    if raw.size % (dim + 1):
        raise ValueError(f"{path}: {raw.size} floats is not a whole number of {dim + 1}-float records")
    rec = raw.reshape(-1, dim + 1)
    return np.ascontiguousarray(rec[:, :dim]), np.ascontiguousarray(rec[:, dim])


def write_point_cloud(path: str | os.PathLike, coords: np.ndarray, alpha: np.ndarray) -> None:
    coords = np.asarray(coords, dtype=np.float32)
    alpha = np.asarray(alpha, dtype=np.float32).reshape(-1, 1)
    if coords.ndim != 2 or coords.shape[1] not in (2, 3) or alpha.shape[0] != coords.shape[0]:
        raise ValueError("coords must be (N, 2) or (N, 3) and alpha (N,)")
    np.concatenate([coords, alpha], axis=1).astype("<f4").tofile(path)


def write_elems_txt(path: str | os.PathLike, elems: np.ndarray) -> None:
    elems = np.asarray(elems, dtype=np.uint32)
    if elems.ndim != 2 or elems.shape[1] not in (3, 4):
        raise ValueError("elems must be (M, 3) triangles or (M, 4) tetrahedra")
    np.savetxt(path, elems, fmt="%u", delimiter=" ")


def read_elems_txt(path: str | os.PathLike, dim: int) -> np.ndarray:
    a = np.loadtxt(path, dtype=np.uint64, ndmin=2)
    if a.size == 0:
        return np.zeros((0, dim + 1), np.uint32)
    if a.shape[1] != dim + 1:
        raise ValueError(f"{path}: expected {dim + 1} ids per line")
    return a.astype(np.uint32)


def write_nodes_txt(path: str | os.PathLike, nodes: np.ndarray) -> None:
    nodes = np.asarray(nodes, dtype=np.float32)
    if nodes.ndim != 2 or nodes.shape[1] not in (2, 3):
        raise ValueError("nodes must be (N, 2) or (N, 3)")
    # the harness prints the float promoted to double with "%.5f"
    np.savetxt(path, nodes.astype(np.float64), fmt="%.5f", delimiter=" ")


def read_nodes_txt(path: str | os.PathLike, dim: int) -> np.ndarray:
    a = np.loadtxt(path, dtype=np.float64, ndmin=2)
    if a.size and a.shape[1] != dim:
        raise ValueError(f"{path}: expected {dim} coordinates per line")
    return a.reshape(-1, dim)


def mesh_point_cloud(path: str | os.PathLike, dim: int, out_dir: str | os.PathLike | None = None):
    """Alpha shape of a .bin point cloud on the GPU, as the reference's
    ``run_on_simulation_meshes.py`` does with its Python API: returns
    (elems, Morton-ordered nodes); with ``out_dir`` also writes ``elems.txt``
    and ``nodes.txt`` there in the harness format."""
    coords, alpha = read_point_cloud(path, dim)
    from .mesh import AlphaShape2D, AlphaShape3D
    a = AlphaShape2D() if dim == 2 else AlphaShape3D()
    a.set_nodes(coords, alpha)
    a.compute()
    elems, nodes = a.get_elem(), a.get_ordered_nodes()
    if out_dir is not None:
        write_elems_txt(os.path.join(out_dir, "elems.txt"), elems)
        write_nodes_txt(os.path.join(out_dir, "nodes.txt"), nodes)
    return elems, nodes
