"""2D alpha shape, same Python surface as the reference's ``stream.mesh.ashape2D``
(python/mesh/ashape2D.py:27-108): ``set_nodes`` (which also runs ``init``),
``init``, ``compute``, ``get_elem``, ``get_ordered_nodes``, over the same C ABI
(src/mesh/DirectAlphaShape2D.cpp:698-753).  Additive methods expose the
permutation, edges, boundary flags and status, which the reference keeps
C++-only (include/mesh/DirectAlphaShape2D.hpp:249-278).
"""
from __future__ import annotations

import ctypes

import numpy as np
import numpy.typing as npt

from .. import check, libmesh

AlphaShape2D_ptr = ctypes.c_void_p
_f32_2d = np.ctypeslib.ndpointer(dtype=np.float32, ndim=2, flags=("C", "ALIGNED"))
_f32_1d = np.ctypeslib.ndpointer(dtype=np.float32, ndim=1, flags=("C", "ALIGNED"))
_u32_2d_w = np.ctypeslib.ndpointer(dtype=np.uint32, ndim=2, flags=("C", "ALIGNED", "WRITEABLE"))
_f32_2d_w = np.ctypeslib.ndpointer(dtype=np.float32, ndim=2, flags=("C", "ALIGNED", "WRITEABLE"))

AlphaShape2D_create = libmesh.AlphaShape2D_create
AlphaShape2D_create.restype = AlphaShape2D_ptr
AlphaShape2D_create.argtypes = []
AlphaShape2D_destroy = libmesh.AlphaShape2D_destroy
AlphaShape2D_destroy.restype = None
AlphaShape2D_destroy.argtypes = [AlphaShape2D_ptr]
AlphaShape2D_set_nodes = libmesh.AlphaShape2D_set_nodes
AlphaShape2D_set_nodes.restype = None
AlphaShape2D_set_nodes.argtypes = [AlphaShape2D_ptr, ctypes.c_uint32, _f32_2d, _f32_1d]
AlphaShape2D_init = libmesh.AlphaShape2D_init
AlphaShape2D_init.restype = None
AlphaShape2D_init.argtypes = [AlphaShape2D_ptr]
AlphaShape2D_compute = libmesh.AlphaShape2D_compute
AlphaShape2D_compute.restype = None
AlphaShape2D_compute.argtypes = [AlphaShape2D_ptr]
AlphaShape2D_get_nelem = libmesh.AlphaShape2D_get_nelem
AlphaShape2D_get_nelem.restype = ctypes.c_uint32
AlphaShape2D_get_nelem.argtypes = [AlphaShape2D_ptr]
AlphaShape2D_get_elem = libmesh.AlphaShape2D_get_elem
AlphaShape2D_get_elem.restype = None
AlphaShape2D_get_elem.argtypes = [AlphaShape2D_ptr, _u32_2d_w]
AlphaShape2D_get_ordered_nodes = libmesh.AlphaShape2D_get_ordered_nodes
AlphaShape2D_get_ordered_nodes.restype = None
AlphaShape2D_get_ordered_nodes.argtypes = [AlphaShape2D_ptr, _f32_2d_w]

_P = ctypes.c_void_p
for _name, _res, _args in [
    ("AlphaShape2D_set_nodes_device", ctypes.c_int, [AlphaShape2D_ptr, ctypes.c_uint32, _P]),
    ("AlphaShape2D_get_status", ctypes.c_int, [AlphaShape2D_ptr]),
    ("AlphaShape2D_get_counters", ctypes.c_int, [AlphaShape2D_ptr, _P]),
    ("AlphaShape2D_get_permutation", ctypes.c_uint32, [AlphaShape2D_ptr, _P]),
    ("AlphaShape2D_get_nedge", ctypes.c_uint32, [AlphaShape2D_ptr]),
    ("AlphaShape2D_get_edges", ctypes.c_uint32, [AlphaShape2D_ptr, _P, _P, _P]),
    ("AlphaShape2D_get_boundary_nodes", ctypes.c_uint32, [AlphaShape2D_ptr, _P]),
    ("AlphaShape2D_get_stars", ctypes.c_int, [AlphaShape2D_ptr, _P, _P, _P, ctypes.c_uint32]),
    ("AlphaShape2D_set_profiling", ctypes.c_int, [AlphaShape2D_ptr, ctypes.c_int]),
    ("AlphaShape2D_get_profile", ctypes.c_int, [AlphaShape2D_ptr, _P]),
    ("AlphaShape2D_synchronize", ctypes.c_int, [AlphaShape2D_ptr]),
]:
    _fn = getattr(libmesh, _name)
    _fn.restype = _res
    _fn.argtypes = _args

STATUS_BITS = {
    0x1: "stack_overflow", 0x8: "tri_cap", 0x10: "exact_overflow", 0x20: "lookback_timeout",
    0x80: "bad_input", 0x100: "cuda_error",
}
# Bits that make compute() raise.  tri_cap marks a star whose local triangle
# list would outgrow its slots (where the reference writes out of bounds): the
# library stops adding to that star and reports the bit.
ERROR_BITS = 0x1 | 0x10 | 0x20 | 0x80 | 0x100
PROFILE_STAGES = ("lbvh", "count_pass", "fill_pass", "star", "scan", "compress")


def _p(a: np.ndarray):
    return a.ctypes.data_as(_P)


class AlphaShape2D:
    """Alpha shape of a 2D point cloud with per-point alpha radii."""

    def __init__(self):
        self.mesh = AlphaShape2D_create()
        if not self.mesh:
            raise MemoryError("AlphaShape2D_create failed")
        self.nnodes = 0

    def __del__(self, _destroy=AlphaShape2D_destroy):  # bound at definition: module globals are gone at exit
        m = getattr(self, "mesh", None)
        if m:
            _destroy(m)
            self.mesh = None

    # ---- reference surface -----------------------------------------------------
    def set_nodes(self, nodes: npt.NDArray[np.float32], alpha: npt.NDArray[np.float32]) -> None:
        nodes = np.ascontiguousarray(nodes, dtype=np.float32)
        alpha = np.ascontiguousarray(alpha, dtype=np.float32)
        if nodes.ndim != 2 or nodes.shape[1] != 2 or alpha.shape != (nodes.shape[0],):
            raise ValueError("nodes must be (N, 2) and alpha (N,)")
        self.nnodes = nodes.shape[0]
        AlphaShape2D_set_nodes(self.mesh, self.nnodes, nodes, alpha)
        self._raise_on_error("set_nodes")
        self.init()

    def init(self) -> None:
        AlphaShape2D_init(self.mesh)
        self._raise_on_error("init")

    def compute(self) -> None:
        AlphaShape2D_compute(self.mesh)
        self._raise_on_error("compute")

    def get_elem(self) -> npt.NDArray[np.uint32]:
        nelems = AlphaShape2D_get_nelem(self.mesh)
        elems = np.empty((nelems, 3), dtype=np.uint32)
        if nelems:
            AlphaShape2D_get_elem(self.mesh, elems)
        return elems

    def get_ordered_nodes(self) -> npt.NDArray[np.float32]:
        nodes = np.empty((self.nnodes, 2), dtype=np.float32)
        AlphaShape2D_get_ordered_nodes(self.mesh, nodes)
        return nodes

    # ---- additive --------------------------------------------------------------
    @property
    def status(self) -> int:
        return int(libmesh.AlphaShape2D_get_status(self.mesh))

    def counters(self) -> dict:
        c = np.zeros(3, np.uint32)
        check(libmesh.AlphaShape2D_get_counters(self.mesh, _p(c)), "get_counters")
        return dict(status=int(c[0]), fill_limited=int(c[1]), exact_calls=int(c[2]))

    def _raise_on_error(self, what: str) -> None:
        st = self.status
        if st & ERROR_BITS:
            from .. import StreamError, last_error
            names = [v for k, v in STATUS_BITS.items() if st & k]
            raise StreamError(f"AlphaShape2D.{what}: status {names}: {last_error()}")

    def get_permutation(self) -> npt.NDArray[np.uint32]:
        """perm[i] = input index of Morton-ordered point i."""
        perm = np.empty(self.nnodes, np.uint32)
        libmesh.AlphaShape2D_get_permutation(self.mesh, _p(perm))
        return perm

    def get_edges(self):
        """CSR adjacency of the alpha shape: (row[n+1], neig[E], edge_is_bnd[E])."""
        ne = libmesh.AlphaShape2D_get_nedge(self.mesh)
        row = np.empty(self.nnodes + 1, np.uint32)
        neig = np.empty(max(ne, 1), np.uint32)
        bnd = np.empty(max(ne, 1), np.uint8)
        libmesh.AlphaShape2D_get_edges(self.mesh, _p(row), _p(neig), _p(bnd))
        return row, neig[:ne], bnd[:ne]

    def get_boundary_nodes(self) -> npt.NDArray[np.uint8]:
        out = np.empty(self.nnodes, np.uint8)
        libmesh.AlphaShape2D_get_boundary_nodes(self.mesh, _p(out))
        return out

    def get_stars(self, width: int | None = None):
        """(nineig[n], nkeep[n], cand[n, width]) in Morton order (diagnostics);
        width defaults to the largest neighbour count."""
        n = self.nnodes
        nineig = np.empty(n, np.uint32)
        nkeep = np.empty(n, np.uint8)
        check(libmesh.AlphaShape2D_get_stars(self.mesh, _p(nineig), _p(nkeep), None, 0), "get_stars")
        if width is None:
            width = int(max(1, int(nineig.max(initial=3)) - 3))
        cand = np.empty((n, width), np.uint32)
        check(libmesh.AlphaShape2D_get_stars(self.mesh, None, None, _p(cand), width), "get_stars")
        return nineig, nkeep, cand

    def set_profiling(self, on: bool = True) -> None:
        check(libmesh.AlphaShape2D_set_profiling(self.mesh, int(on)), "set_profiling")

    def profile(self) -> dict:
        ms = np.zeros(len(PROFILE_STAGES), np.float32)
        check(libmesh.AlphaShape2D_get_profile(self.mesh, _p(ms)), "get_profile")
        return {k: float(v) for k, v in zip(PROFILE_STAGES, ms)}
