"""2D Delaunay mesher, same Python surface as the reference's ``stream.mesh.mesh``
(python/mesh/mesh.py:86-136): ``set_nodes`` (which also runs ``init``),
``insert_morton_neighbors``, ``insert_BVH_neighbors``, ``insert_iterative``,
``remove_super_nodes``, ``get_elem``, ``get_ordered_nodes``, over the same C
ABI (src/mesh/mesh.cpp:806-862).  Additive methods expose the permutation,
the super nodes and the status.
"""
from __future__ import annotations

import ctypes

import numpy as np
import numpy.typing as npt

from .. import check, libmesh

mesh2D_ptr = ctypes.c_void_p
_f32_2d = np.ctypeslib.ndpointer(dtype=np.float32, ndim=2, flags=("C", "ALIGNED"))
_u32_2d_w = np.ctypeslib.ndpointer(dtype=np.uint32, ndim=2, flags=("C", "ALIGNED", "WRITEABLE"))
_f32_2d_w = np.ctypeslib.ndpointer(dtype=np.float32, ndim=2, flags=("C", "ALIGNED", "WRITEABLE"))
_P = ctypes.c_void_p

for _name, _res, _args in [
    ("Mesh2D_create", mesh2D_ptr, []),
    ("Mesh2D_destroy", None, [mesh2D_ptr]),
    ("Mesh2D_set_nodes", None, [mesh2D_ptr, ctypes.c_uint32, _f32_2d]),
    ("Mesh2D_init", None, [mesh2D_ptr]),
    ("Mesh2D_insert_morton_neighbors", None, [mesh2D_ptr]),
    ("Mesh2D_insert_BVH_neighbors", None, [mesh2D_ptr]),
    ("Mesh2D_insert_iterative", None, [mesh2D_ptr]),
    ("Mesh2D_remove_super_nodes", None, [mesh2D_ptr]),
    ("Mesh2D_get_nelem", ctypes.c_uint32, [mesh2D_ptr]),
    ("Mesh2D_get_elem", None, [mesh2D_ptr, _u32_2d_w]),
    ("Mesh2D_get_ordered_nodes", None, [mesh2D_ptr, _f32_2d_w]),
    ("Mesh2D_get_status", ctypes.c_int, [mesh2D_ptr]),
    ("Mesh2D_get_counters", ctypes.c_int, [mesh2D_ptr, _P]),
    ("Mesh2D_get_permutation", ctypes.c_uint32, [mesh2D_ptr, _P]),
    ("Mesh2D_get_super_nodes", ctypes.c_int, [mesh2D_ptr, _P]),
]:
    _fn = getattr(libmesh, _name)
    _fn.restype = _res
    _fn.argtypes = _args

STATUS_BITS = {
    0x1: "stack_overflow", 0x2: "query_budget", 0x8: "local_id_cap", 0x10: "exact_overflow",
    0x20: "lookback_timeout", 0x80: "bad_input", 0x100: "cuda_error", 0x200: "incomplete",
}
# Bits that make a call raise (query_budget, local_id_cap and incomplete are
# reported by status / counters(): the stars concerned stay unverified).
ERROR_BITS = 0x1 | 0x10 | 0x20 | 0x80 | 0x100


class Mesh2D:
    """Delaunay triangulation of a 2D point cloud (with three super nodes)."""

    def __init__(self):
        self.mesh = libmesh.Mesh2D_create()
        if not self.mesh:
            raise MemoryError("Mesh2D_create failed")
        self.nnodes = 0

    def __del__(self, _destroy=libmesh.Mesh2D_destroy):  # bound at definition: module globals are gone at exit
        m = getattr(self, "mesh", None)
        if m:
            _destroy(m)
            self.mesh = None

    # ---- reference surface -----------------------------------------------------
    def init(self) -> None:
        libmesh.Mesh2D_init(self.mesh)
        self._raise_on_error("init")

    def set_nodes(self, nodes: npt.NDArray[np.float32]) -> None:
        nodes = np.ascontiguousarray(nodes, dtype=np.float32)
        if nodes.ndim != 2 or nodes.shape[1] != 2:
            raise ValueError("nodes must be (N, 2)")
        self.nnodes = nodes.shape[0]
        libmesh.Mesh2D_set_nodes(self.mesh, self.nnodes, nodes)
        self._raise_on_error("set_nodes")
        self.init()

    def insert_morton_neighbors(self) -> None:
        libmesh.Mesh2D_insert_morton_neighbors(self.mesh)
        self._raise_on_error("insert_morton_neighbors")

    def insert_BVH_neighbors(self) -> None:  # noqa: N802  (the reference's name)
        libmesh.Mesh2D_insert_BVH_neighbors(self.mesh)
        self._raise_on_error("insert_BVH_neighbors")

    def insert_iterative(self) -> None:
        libmesh.Mesh2D_insert_iterative(self.mesh)
        self._raise_on_error("insert_iterative")

    def remove_super_nodes(self) -> None:
        libmesh.Mesh2D_remove_super_nodes(self.mesh)

    def get_elem(self) -> npt.NDArray[np.uint32]:
        nelems = libmesh.Mesh2D_get_nelem(self.mesh)
        self._raise_on_error("get_nelem")
        elems = np.empty((nelems, 3), dtype=np.uint32)
        if nelems:
            libmesh.Mesh2D_get_elem(self.mesh, elems)
        return elems

    def get_ordered_nodes(self) -> npt.NDArray[np.float32]:
        nodes = np.empty((self.nnodes, 2), dtype=np.float32)
        libmesh.Mesh2D_get_ordered_nodes(self.mesh, nodes)
        return nodes

    # ---- additive --------------------------------------------------------------
    @property
    def status(self) -> int:
        return int(libmesh.Mesh2D_get_status(self.mesh))

    def counters(self) -> dict:
        c = np.zeros(2, np.uint32)
        check(libmesh.Mesh2D_get_counters(self.mesh, c.ctypes.data_as(_P)), "get_counters")
        return dict(status=int(c[0]), incomplete=int(c[1]))

    def get_permutation(self) -> npt.NDArray[np.uint32]:
        """perm[i] = input index of Morton-ordered point i."""
        perm = np.empty(self.nnodes, np.uint32)
        libmesh.Mesh2D_get_permutation(self.mesh, perm.ctypes.data_as(_P))
        return perm

    def get_super_nodes(self) -> npt.NDArray[np.float32]:
        xy = np.empty((3, 2), np.float32)
        check(libmesh.Mesh2D_get_super_nodes(self.mesh, xy.ctypes.data_as(_P)), "get_super_nodes")
        return xy

    def _raise_on_error(self, what: str) -> None:
        st = self.status
        if st & ERROR_BITS:
            from .. import StreamError, last_error
            names = [v for k, v in STATUS_BITS.items() if st & k]
            raise StreamError(f"Mesh2D.{what}: status {names}: {last_error()}")
