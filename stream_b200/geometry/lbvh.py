"""Karras LBVH over 3D spheres (the reference's ``Sphere3DLBVH``,
include/geometry/lbvh.hpp:50,62-362), through the library's C boundary."""
from __future__ import annotations

import ctypes

import numpy as np

from .. import check, libgeo

_P = ctypes.c_void_p
for _name, _res, _args in [
    ("Sphere3DLBVH_create", _P, []),
    ("Sphere3DLBVH_destroy", None, [_P]),
    ("Sphere3DLBVH_set_objects", ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_int, ctypes.c_int]),
    ("Sphere3DLBVH_set_objects_device", ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_int, ctypes.c_int]),
    ("Sphere3DLBVH_build", ctypes.c_int, [_P]),
    ("Sphere3DLBVH_synchronize", ctypes.c_int, [_P, _P]),
    ("Sphere3DLBVH_get", ctypes.c_int, [_P] + [_P] * 9),
    ("Sphere3DLBVH_set_profiling", ctypes.c_int, [_P, ctypes.c_int]),
    ("Sphere3DLBVH_get_profile", ctypes.c_uint32, [_P, _P, ctypes.c_uint32]),
]:
    _fn = getattr(libgeo, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class Sphere3DLBVH:
    """LBVH over spheres given as an (n, 4) float32 array (x, y, z, r)."""

    def __init__(self):
        self.h = libgeo.Sphere3DLBVH_create()
        if not self.h:
            raise MemoryError("Sphere3DLBVH_create failed")
        self.n = 0

    def __del__(self, _destroy=libgeo.Sphere3DLBVH_destroy):  # bound at definition: module globals are gone at exit
        h = getattr(self, "h", None)
        if h:
            _destroy(h)
            self.h = None

    def set_objects_device(self, d_xyzr: int, n: int, bits: int = 63, fit_point: bool = False) -> None:
        """Objects already on the device: d_xyzr is the address of n x 4 float32 (x, y, z, r)."""
        self.n = int(n)
        check(libgeo.Sphere3DLBVH_set_objects_device(self.h, self.n, _P(d_xyzr), bits, int(fit_point)),
              "Sphere3DLBVH_set_objects_device")

    def set_objects(self, xyzr: np.ndarray, bits: int = 63, fit_point: bool = False) -> None:
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        if xyzr.ndim != 2 or xyzr.shape[1] != 4:
            raise ValueError("xyzr must be (n, 4)")
        self.n = xyzr.shape[0]
        check(libgeo.Sphere3DLBVH_set_objects(self.h, self.n, xyzr.ctypes.data_as(_P), bits, int(fit_point)),
              "Sphere3DLBVH_set_objects")

    def build(self) -> int:
        check(libgeo.Sphere3DLBVH_build(self.h), "Sphere3DLBVH_build")
        st = ctypes.c_uint32()
        check(libgeo.Sphere3DLBVH_synchronize(self.h, ctypes.byref(st)), "Sphere3DLBVH_synchronize")
        return int(st.value)

    STAGES = ("bbox_morton_hist", "radix_sort", "gather", "karras_fit")

    def set_profiling(self, on: bool = True) -> None:
        check(libgeo.Sphere3DLBVH_set_profiling(self.h, int(on)), "Sphere3DLBVH_set_profiling")

    def profile(self) -> dict:
        """Stage times (ms) of the last build made with profiling on."""
        ms = np.zeros(8, np.float32)
        k = libgeo.Sphere3DLBVH_get_profile(self.h, ms.ctypes.data_as(_P), 8)
        return {name: float(v) for name, v in zip(self.STAGES, ms[:k])}

    def arrays(self) -> dict:
        n = self.n
        out = dict(
            bb_glob=np.zeros(6, np.float32), morton=np.zeros(n, np.uint64), perm=np.zeros(n, np.uint32),
            sep=np.zeros(n - 1, np.int32), cil=np.zeros(n - 1, np.uint8), leaf_parent=np.zeros(n, np.uint32),
            internal_parent=np.zeros(n - 1, np.uint32), bboxes=np.zeros((n - 1, 6), np.float32),
            obj_m=np.zeros((n, 4), np.float32))
        check(libgeo.Sphere3DLBVH_get(self.h, *[out[k].ctypes.data_as(_P) for k in (
            "bb_glob", "morton", "perm", "sep", "cil", "leaf_parent", "internal_parent", "bboxes", "obj_m")]),
            "Sphere3DLBVH_get")
        return out


for _name, _res, _args in [
    ("Sphere3DTRBVH_create", _P, []),
    ("Sphere3DTRBVH_destroy", None, [_P]),
    ("Sphere3DTRBVH_set_objects", ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("Sphere3DTRBVH_build", ctypes.c_int, [_P]),
    ("Sphere3DTRBVH_synchronize", ctypes.c_int, [_P, _P]),
    ("Sphere3DTRBVH_get", ctypes.c_int, [_P] + [_P] * 10),
    ("Sphere3DTRBVH_count_overlaps", ctypes.c_int, [_P, _P]),
    ("Sphere3DTRBVH_set_profiling", ctypes.c_int, [_P, ctypes.c_int]),
    ("Sphere3DTRBVH_get_profile", ctypes.c_uint32, [_P, _P, ctypes.c_uint32]),
]:
    _fn = getattr(libgeo, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class Sphere3DTRBVH:
    """TRBVH over spheres (the reference's ``Sphere3DTRBVH``,
    include/geometry/trbvh.hpp:55): Apetrei build + treelet restructuring."""

    def __init__(self):
        self.h = libgeo.Sphere3DTRBVH_create()
        if not self.h:
            raise MemoryError("Sphere3DTRBVH_create failed")
        self.n = 0

    def __del__(self, _destroy=libgeo.Sphere3DTRBVH_destroy):  # bound at definition: module globals are gone at exit
        h = getattr(self, "h", None)
        if h:
            _destroy(h)
            self.h = None

    def set_objects(self, xyzr: np.ndarray, treelet_size: int = 7, area3d: bool = True, rounds: int = 3) -> None:
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        if xyzr.ndim != 2 or xyzr.shape[1] != 4:
            raise ValueError("xyzr must be (n, 4)")
        self.n = xyzr.shape[0]
        check(libgeo.Sphere3DTRBVH_set_objects(self.h, self.n, xyzr.ctypes.data_as(_P), treelet_size, int(area3d),
                                               rounds), "Sphere3DTRBVH_set_objects")

    def build(self) -> int:
        check(libgeo.Sphere3DTRBVH_build(self.h), "Sphere3DTRBVH_build")
        st = ctypes.c_uint32()
        check(libgeo.Sphere3DTRBVH_synchronize(self.h, ctypes.byref(st)), "Sphere3DTRBVH_synchronize")
        return int(st.value)

    def arrays(self) -> dict:
        n = self.n
        m = 2 * n - 1
        out = dict(child_left=np.zeros(n - 1, np.uint32), child_right=np.zeros(n - 1, np.uint32),
                   range_min=np.zeros(n - 1, np.uint32), range_max=np.zeros(n - 1, np.uint32),
                   parent=np.zeros(m, np.uint32), bboxes=np.zeros((m, 6), np.float32),
                   subtree_size=np.zeros(m, np.uint32), sah=np.zeros(m, np.float32), root=np.zeros(1, np.uint32),
                   obj_m=np.zeros((n, 4), np.float32))
        check(libgeo.Sphere3DTRBVH_get(self.h, *[out[k].ctypes.data_as(_P) for k in (
            "child_left", "child_right", "range_min", "range_max", "parent", "bboxes", "subtree_size", "sah", "root",
            "obj_m")]), "Sphere3DTRBVH_get")
        out["root"] = int(out["root"][0])
        return out

    STAGES = ("bbox_morton_hist", "radix_sort", "gather", "apetrei", "treelets")

    def set_profiling(self, on: bool = True) -> None:
        check(libgeo.Sphere3DTRBVH_set_profiling(self.h, int(on)), "Sphere3DTRBVH_set_profiling")

    def profile(self) -> dict:
        """Stage times (ms) of the last build made with profiling on."""
        ms = np.zeros(8, np.float32)
        k = libgeo.Sphere3DTRBVH_get_profile(self.h, ms.ctypes.data_as(_P), 8)
        return {name: float(v) for name, v in zip(self.STAGES, ms[:k])}

    def count_overlaps(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        check(libgeo.Sphere3DTRBVH_count_overlaps(self.h, out.ctypes.data_as(_P)), "count_overlaps")
        return out


class Sphere3DLBVHa:
    """The reference's LBVHa (include/geometry/lbvh_agglo.hpp:63-361): Apetrei's
    agglomerative LBVH over 3D spheres, bottom-up from the sorted 63-bit
    Morton codes.  It is the TRBVH build without restructuring rounds (the
    same kernels); arrays in the reference's layout: children[n-1][2],
    range[n-1][2], parent[2n-1] (leaves 0..n-1, internal nodes n..2n-2, root
    parent 2n), bboxes[2n-1][6], root, obj_m[n][4]."""

    def __init__(self):
        self._t = Sphere3DTRBVH()
        self.n = 0

    def set_objects(self, xyzr: np.ndarray) -> None:
        self._t.set_objects(xyzr, treelet_size=5, area3d=False, rounds=0)
        self.n = self._t.n

    def build(self) -> int:
        return self._t.build()

    def arrays(self) -> dict:
        a = self._t.arrays()
        return dict(children=np.stack([a["child_left"], a["child_right"]], 1),
                    range=np.stack([a["range_min"], a["range_max"]], 1), parent=a["parent"], bboxes=a["bboxes"],
                    root=a["root"], obj_m=a["obj_m"])
