"""3D alpha shape, same Python surface as the reference's ``stream.mesh.ashape3D``
(python/mesh/ashape3D.py:27-110): ``set_nodes`` (which also runs ``init``),
``init``, ``compute``, ``get_elem``, ``get_ordered_nodes``, over the same C ABI
(src/mesh/DirectAlphaShape3D.cpp:754-810).  Additive methods expose the
permutation, edges, free-surface flags and status, which the reference keeps
C++-only (include/mesh/DirectAlphaShape3D.hpp:186-236).
"""
from __future__ import annotations

import ctypes

import numpy as np
import numpy.typing as npt

from .. import check, libmesh

AlphaShape3D_ptr = ctypes.c_void_p
_f32_2d = np.ctypeslib.ndpointer(dtype=np.float32, ndim=2, flags=("C", "ALIGNED"))
_f32_1d = np.ctypeslib.ndpointer(dtype=np.float32, ndim=1, flags=("C", "ALIGNED"))
_u32_2d_w = np.ctypeslib.ndpointer(dtype=np.uint32, ndim=2, flags=("C", "ALIGNED", "WRITEABLE"))
_f32_2d_w = np.ctypeslib.ndpointer(dtype=np.float32, ndim=2, flags=("C", "ALIGNED", "WRITEABLE"))

AlphaShape3D_create = libmesh.AlphaShape3D_create
AlphaShape3D_create.restype = AlphaShape3D_ptr
AlphaShape3D_create.argtypes = []
AlphaShape3D_destroy = libmesh.AlphaShape3D_destroy
AlphaShape3D_destroy.restype = None
AlphaShape3D_destroy.argtypes = [AlphaShape3D_ptr]
AlphaShape3D_set_nodes = libmesh.AlphaShape3D_set_nodes
AlphaShape3D_set_nodes.restype = None
AlphaShape3D_set_nodes.argtypes = [AlphaShape3D_ptr, ctypes.c_uint32, _f32_2d, _f32_1d]
AlphaShape3D_init = libmesh.AlphaShape3D_init
AlphaShape3D_init.restype = None
AlphaShape3D_init.argtypes = [AlphaShape3D_ptr]
AlphaShape3D_compute = libmesh.AlphaShape3D_compute
AlphaShape3D_compute.restype = None
AlphaShape3D_compute.argtypes = [AlphaShape3D_ptr]
AlphaShape3D_get_nelem = libmesh.AlphaShape3D_get_nelem
AlphaShape3D_get_nelem.restype = ctypes.c_uint32
AlphaShape3D_get_nelem.argtypes = [AlphaShape3D_ptr]
AlphaShape3D_get_elem = libmesh.AlphaShape3D_get_elem
AlphaShape3D_get_elem.restype = None
AlphaShape3D_get_elem.argtypes = [AlphaShape3D_ptr, _u32_2d_w]
AlphaShape3D_get_ordered_nodes = libmesh.AlphaShape3D_get_ordered_nodes
AlphaShape3D_get_ordered_nodes.restype = None
AlphaShape3D_get_ordered_nodes.argtypes = [AlphaShape3D_ptr, _f32_2d_w]

_P = ctypes.c_void_p
for _name, _res, _args in [
    ("AlphaShape3D_set_morton_bits", ctypes.c_int, [AlphaShape3D_ptr, ctypes.c_int]),
    ("AlphaShape3D_set_nodes_device", ctypes.c_int, [AlphaShape3D_ptr, ctypes.c_uint32, _P]),
    ("AlphaShape3D_get_status", ctypes.c_int, [AlphaShape3D_ptr]),
    ("AlphaShape3D_get_counters", ctypes.c_int, [AlphaShape3D_ptr, _P]),
    ("AlphaShape3D_get_permutation", ctypes.c_uint32, [AlphaShape3D_ptr, _P]),
    ("AlphaShape3D_get_nedge", ctypes.c_uint32, [AlphaShape3D_ptr]),
    ("AlphaShape3D_get_edges", ctypes.c_uint32, [AlphaShape3D_ptr, _P, _P, _P]),
    ("AlphaShape3D_get_boundary_nodes", ctypes.c_uint32, [AlphaShape3D_ptr, _P]),
    ("AlphaShape3D_get_stars", ctypes.c_int, [AlphaShape3D_ptr, _P, _P, _P]),
    ("AlphaShape3D_synchronize", ctypes.c_int, [AlphaShape3D_ptr]),
]:
    _fn = getattr(libmesh, _name)
    _fn.restype = _res
    _fn.argtypes = _args

STATUS_BITS = {
    0x1: "stack_overflow", 0x2: "walk_cap", 0x4: "broken_cycle", 0x8: "tet_cap",
    0x10: "exact_overflow", 0x20: "lookback_timeout", 0x40: "truncated", 0x80: "bad_input",
    0x100: "cuda_error",
}
# Bits that make compute() raise: the result is not trustworthy.  walk_cap
# and truncated are reference behaviour (reported only); broken_cycle and
# tet_cap mark stars where the reference itself reads or writes out of bounds
# (undefined behaviour, e.g. exactly duplicated points): the library stops
# inserting into that star, reports the bit, and the rest of the output stands.
ERROR_BITS = 0x1 | 0x10 | 0x20 | 0x80 | 0x100


def _p(a: np.ndarray):
    return a.ctypes.data_as(_P)


class AlphaShape3D:
    """Alpha shape of a 3D point cloud with per-point alpha radii."""

    def __init__(self, morton_bits: int = 63):
        self.mesh = AlphaShape3D_create()
        if not self.mesh:
            raise MemoryError("AlphaShape3D_create failed")
        self.nnodes = 0
        if morton_bits != 63:
            check(libmesh.AlphaShape3D_set_morton_bits(self.mesh, morton_bits), "set_morton_bits")

    def __del__(self, _destroy=AlphaShape3D_destroy):  # bound at definition: module globals are gone at exit
        m = getattr(self, "mesh", None)
        if m:
            _destroy(m)
            self.mesh = None

    # ---- reference surface -----------------------------------------------------
    def set_nodes(self, nodes: npt.NDArray[np.float32], alpha: npt.NDArray[np.float32]) -> None:
        nodes = np.ascontiguousarray(nodes, dtype=np.float32)
        alpha = np.ascontiguousarray(alpha, dtype=np.float32)
        if nodes.ndim != 2 or nodes.shape[1] != 3 or alpha.shape != (nodes.shape[0],):
            raise ValueError("nodes must be (N, 3) and alpha (N,)")
        self.nnodes = nodes.shape[0]
        AlphaShape3D_set_nodes(self.mesh, self.nnodes, nodes, alpha)
        self._raise_on_error("set_nodes")
        self.init()

    def init(self) -> None:
        AlphaShape3D_init(self.mesh)
        self._raise_on_error("init")

    def compute(self) -> None:
        AlphaShape3D_compute(self.mesh)
        self._raise_on_error("compute")

    def get_elem(self) -> npt.NDArray[np.uint32]:
        nelems = AlphaShape3D_get_nelem(self.mesh)
        elems = np.empty((nelems, 4), dtype=np.uint32)
        if nelems:
            AlphaShape3D_get_elem(self.mesh, elems)
        return elems

    def get_ordered_nodes(self) -> npt.NDArray[np.float32]:
        nodes = np.empty((self.nnodes, 3), dtype=np.float32)
        AlphaShape3D_get_ordered_nodes(self.mesh, nodes)
        return nodes

    # ---- additive --------------------------------------------------------------
    @property
    def status(self) -> int:
        return int(libmesh.AlphaShape3D_get_status(self.mesh))

    def counters(self) -> dict:
        c = np.zeros(4, np.uint32)
        check(libmesh.AlphaShape3D_get_counters(self.mesh, _p(c)), "get_counters")
        return dict(status=int(c[0]), deferred=int(c[1]), truncated=int(c[2]), exact_calls=int(c[3]))

    def _raise_on_error(self, what: str) -> None:
        st = self.status
        if st & ERROR_BITS:
            from .. import StreamError, last_error
            names = [v for k, v in STATUS_BITS.items() if st & k]
            raise StreamError(f"AlphaShape3D.{what}: status {names}: {last_error()}")

    def get_permutation(self) -> npt.NDArray[np.uint32]:
        """perm[i] = input index of Morton-ordered point i."""
        perm = np.empty(self.nnodes, np.uint32)
        libmesh.AlphaShape3D_get_permutation(self.mesh, _p(perm))
        return perm

    def get_edges(self):
        """CSR adjacency of the alpha shape: (row[n+1], neig[E], edge_is_bnd[E])."""
        ne = libmesh.AlphaShape3D_get_nedge(self.mesh)
        row = np.empty(self.nnodes + 1, np.uint32)
        neig = np.empty(max(ne, 1), np.uint32)
        bnd = np.empty(max(ne, 1), np.uint8)
        libmesh.AlphaShape3D_get_edges(self.mesh, _p(row), _p(neig), _p(bnd))
        return row, neig[:ne], bnd[:ne]

    def get_boundary_nodes(self) -> npt.NDArray[np.uint8]:
        out = np.empty(self.nnodes, np.uint8)
        libmesh.AlphaShape3D_get_boundary_nodes(self.mesh, _p(out))
        return out

    def get_stars(self):
        """(nineig[n], nkeep[n], cand[n, 124]) in Morton order (diagnostics)."""
        n = self.nnodes
        nineig = np.empty(n, np.uint32)
        nkeep = np.empty(n, np.uint8)
        cand = np.empty((n, 124), np.uint32)
        check(libmesh.AlphaShape3D_get_stars(self.mesh, _p(nineig), _p(nkeep), _p(cand)), "get_stars")
        return nineig, nkeep, cand
