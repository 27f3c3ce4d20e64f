"""ctypes front end of the oracle (test infrastructure only).

Two checkers live under ``oracle/``:

* ``_build/liboracle.so`` -- the plain-C restatement (``restate/*.c``) of the
  reference's LBVH, 3D and 2D alpha shapes and FP32 CG
  (src/mesh/DirectAlphaShape3D.cpp, src/mesh/DirectAlphaShape2D.cpp,
  include/geometry/lbvh.hpp, src/numerics/conjugate_gradient.cpp).
* ``_ref/libstream_ref.so`` -- the reference's own, unmodified sources compiled
  for the host against ``ava_shim`` (a CPU stand-in for the absent AVA layer).
  Present when it was built where the reference tree exists; it travels with
  the repository copy.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline import
this module.  The product (``stream_b200``) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libstream_ref.so")
# Root of the reference tree, needed only to build _ref (not at test time).
REF_TREE = os.environ.get("STREAM_REFERENCE", "")

P = ctypes.c_void_p
U32 = ctypes.c_uint32


def build(with_ref: bool | None = None) -> None:
    """Compile the restatement, and the reference build when its tree exists."""
    targets = ["restate"]
    if with_ref is None:
        with_ref = bool(REF_TREE) and os.path.isdir(REF_TREE)
    if with_ref:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", HERE, *targets, *([f"REF={REF_TREE}"] if REF_TREE else [])], check=True)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(P)


class _Struct(ctypes.Structure):
    _fields_ = [
        ("n", U32), ("n_elems", U32), ("n_edges", U32), ("status", U32),
        ("n_truncated", U32), ("n_exact", U32),
        ("perm", P), ("coords_m", P), ("nineig", P), ("cand", P), ("elemrow", P),
        ("elems", P), ("row", P), ("neig", P), ("edge_is_bnd", P),
        ("node_is_bnd", P), ("nelem", P),
    ]


class _TrStruct(ctypes.Structure):
    _fields_ = [("n", U32), ("root", U32), ("child_left", P), ("child_right", P), ("range_min", P),
                ("range_max", P), ("parent", P), ("bboxes", P), ("subtree_size", P), ("sah", P), ("obj_m", P)]


@dataclass
class AlphaShapeResult:
    """Outputs of one alpha-shape run, in the reference's Morton-ordered ids."""
    perm: np.ndarray
    coords_m: np.ndarray
    nineig: np.ndarray
    cand: np.ndarray
    elems: np.ndarray
    row: np.ndarray
    neig: np.ndarray
    edge_is_bnd: np.ndarray
    node_is_bnd: np.ndarray
    nelem: np.ndarray
    status: int = 0
    n_truncated: int = 0
    n_exact: int = 0


class _Struct2(ctypes.Structure):
    _fields_ = [
        ("n", U32), ("n_elems", U32), ("n_edges", U32), ("status", U32), ("n_exact", U32),
        ("bb_glob", ctypes.c_float * 4), ("codes", P), ("perm", P), ("coords_m", P), ("nineig", P),
        ("row_offset", P), ("cand", P), ("elemrow", P), ("elems", P), ("row", P), ("neig", P),
        ("edge_is_bnd", P), ("node_is_bnd", P), ("nelem", P),
    ]


@dataclass
class AlphaShape2DResult:
    """Outputs of one 2D alpha-shape run, in the reference's Morton-ordered ids.
    coords_m: (n+3) x 3 (x, y, alpha) incl. the 3 infinity points; cand: n x w
    neighbour rows in traversal order, UINT32_MAX padded."""
    perm: np.ndarray
    coords_m: np.ndarray
    nineig: np.ndarray
    cand: np.ndarray
    elems: np.ndarray
    row: np.ndarray
    neig: np.ndarray
    edge_is_bnd: np.ndarray
    node_is_bnd: np.ndarray
    nelem: np.ndarray
    status: int = 0
    n_exact: int = 0
    bb_glob: np.ndarray | None = None
    morton: np.ndarray | None = None


def _copy(addr, dtype, count):
    if count == 0:
        return np.zeros(0, dtype=dtype)
    buf = (ctypes.c_char * (np.dtype(dtype).itemsize * count)).from_address(addr)
    return np.frombuffer(bytes(buf), dtype=dtype).copy()


class Restatement:
    """The plain-C restatement (always available after ``build()``)."""

    def __init__(self, path: str = RESTATE_SO):
        if not os.path.exists(path):
            build(with_ref=False)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.orc_cg_f32.restype = U32
        L.orc_insphere_filter.restype = ctypes.c_float
        L.orc_insphere_exact.restype = ctypes.c_float
        L.orc_orient3d.restype = ctypes.c_float

    # ---- LBVH --------------------------------------------------------------
    def lbvh3d(self, xyzr: np.ndarray, bits: int = 63, fit_point: bool = False) -> dict:
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        n = xyzr.shape[0]
        out = dict(
            bb_glob=np.zeros(6, np.float32), morton=np.zeros(n, np.uint64),
            perm=np.zeros(n, np.uint32), sep=np.zeros(n - 1, np.int32),
            cil=np.zeros(n - 1, np.uint8), leaf_parent=np.zeros(n, np.uint32),
            internal_parent=np.zeros(n - 1, np.uint32),
            bboxes=np.zeros((n - 1, 6), np.float32), obj_m=np.zeros((n, 4), np.float32))
        self.lib.orc_lbvh3d(U32(n), _ptr(xyzr), ctypes.c_int(bits), ctypes.c_int(int(fit_point)),
                            *[_ptr(out[k]) for k in ("bb_glob", "morton", "perm", "sep", "cil",
                                                     "leaf_parent", "internal_parent", "bboxes",
                                                     "obj_m")])
        return out

    def morton3d(self, xyzr: np.ndarray, bb: np.ndarray, bits: int = 63) -> np.ndarray:
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        bb = np.ascontiguousarray(bb, dtype=np.float32)
        out = np.zeros(xyzr.shape[0], np.uint64)
        self.lib.orc_morton3d(U32(xyzr.shape[0]), _ptr(xyzr), _ptr(bb), ctypes.c_int(bits), _ptr(out))
        return out

    def sort_pairs(self, keys: np.ndarray, vals: np.ndarray):
        k = np.ascontiguousarray(keys, dtype=np.uint64).copy()
        v = np.ascontiguousarray(vals, dtype=np.uint32).copy()
        self.lib.orc_sort_pairs(U32(k.size), _ptr(k), _ptr(v))
        return k, v

    # ---- TRBVH ---------------------------------------------------------------
    def trbvh3d(self, xyzr: np.ndarray, treelet_size: int = 7, area3d: bool = True, rounds: int = 3,
                count: bool = False) -> dict:
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        n = xyzr.shape[0]
        t = _TrStruct()
        if self.lib.orc_trbvh3d(U32(n), _ptr(xyzr), ctypes.c_int(treelet_size), ctypes.c_int(int(area3d)),
                                ctypes.c_int(rounds), ctypes.byref(t)) != 0:
            raise ValueError("orc_trbvh3d: bad arguments")
        try:
            m = 2 * n - 1
            out = dict(root=int(t.root), child_left=_copy(t.child_left, np.uint32, n - 1),
                       child_right=_copy(t.child_right, np.uint32, n - 1),
                       range_min=_copy(t.range_min, np.uint32, n - 1), range_max=_copy(t.range_max, np.uint32, n - 1),
                       parent=_copy(t.parent, np.uint32, m), bboxes=_copy(t.bboxes, np.float32, 6 * m).reshape(m, 6),
                       subtree_size=_copy(t.subtree_size, np.uint32, m), sah=_copy(t.sah, np.float32, m),
                       obj_m=_copy(t.obj_m, np.float32, 4 * n).reshape(n, 4))
            if count:
                c = np.zeros(n, np.uint32)
                self.lib.orc_trbvh3d_count(ctypes.byref(t), _ptr(c))
                out["count"] = c
        finally:
            self.lib.orc_trbvh3d_free(ctypes.byref(t))
        return out

    # ---- alpha shape ---------------------------------------------------------
    def ashape3d(self, coords: np.ndarray, alpha: np.ndarray, bits: int = 63) -> AlphaShapeResult:
        coords = np.ascontiguousarray(coords, dtype=np.float32)
        alpha = np.ascontiguousarray(alpha, dtype=np.float32)
        n = coords.shape[0]
        s = _Struct()
        rc = self.lib.orc_ashape3d(U32(n), _ptr(coords), _ptr(alpha), ctypes.c_int(bits), ctypes.byref(s))
        if rc != 0:
            raise ValueError("oracle alpha shape needs at least 2 points")
        try:
            r = AlphaShapeResult(
                perm=_copy(s.perm, np.uint32, n),
                coords_m=_copy(s.coords_m, np.float32, 4 * (n + 4)).reshape(n + 4, 4),
                nineig=_copy(s.nineig, np.uint32, n),
                cand=_copy(s.cand, np.uint32, 124 * n).reshape(n, 124),
                elems=_copy(s.elems, np.uint32, 4 * s.n_elems).reshape(-1, 4),
                row=_copy(s.row, np.uint32, n + 1),
                neig=_copy(s.neig, np.uint32, s.n_edges),
                edge_is_bnd=_copy(s.edge_is_bnd, np.uint8, s.n_edges),
                node_is_bnd=_copy(s.node_is_bnd, np.uint8, n),
                nelem=_copy(s.nelem, np.uint8, n),
                status=s.status, n_truncated=s.n_truncated, n_exact=s.n_exact)
        finally:
            self.lib.orc_ashape3d_free(ctypes.byref(s))
        return r

    def ashape2d(self, coords: np.ndarray, alpha: np.ndarray) -> AlphaShape2DResult:
        coords = np.ascontiguousarray(coords, dtype=np.float32).reshape(-1, 2)
        alpha = np.ascontiguousarray(alpha, dtype=np.float32)
        n = coords.shape[0]
        s = _Struct2()
        if self.lib.orc_ashape2d(U32(n), _ptr(coords), _ptr(alpha), ctypes.byref(s)) != 0:
            raise ValueError("oracle alpha shape needs at least 2 points")
        try:
            nineig = _copy(s.nineig, np.uint32, n)
            roff = _copy(s.row_offset, np.uint32, n + 1)
            flat = _copy(s.cand, np.uint32, int(roff[-1]))
            k = nineig.astype(np.int64) - 3
            w = int(max(1, k.max(initial=0)))
            cand = np.full((n, w), 0xFFFFFFFF, np.uint32)
            for i in np.nonzero(k > 0)[0]:
                cand[i, :k[i]] = flat[roff[i]:roff[i] + k[i]]
            cm = _copy(s.coords_m, np.float32, 4 * (n + 3)).reshape(n + 3, 4)
            r = AlphaShape2DResult(
                perm=_copy(s.perm, np.uint32, n), coords_m=cm[:, [0, 1, 3]].copy(), nineig=nineig, cand=cand,
                elems=_copy(s.elems, np.uint32, 3 * s.n_elems).reshape(-1, 3),
                row=_copy(s.row, np.uint32, n + 1), neig=_copy(s.neig, np.uint32, s.n_edges),
                edge_is_bnd=_copy(s.edge_is_bnd, np.uint8, s.n_edges),
                node_is_bnd=_copy(s.node_is_bnd, np.uint8, n), nelem=_copy(s.nelem, np.uint8, n),
                status=s.status, n_exact=s.n_exact, bb_glob=np.array(s.bb_glob[:], np.float32),
                morton=_copy(s.codes, np.uint64, n))
        finally:
            self.lib.orc_ashape2d_free(ctypes.byref(s))
        return r

    # ---- predicates ----------------------------------------------------------
    def conflict_batch(self, pts: np.ndarray, ids: np.ndarray):
        pts = np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 5, 3)
        ids = np.ascontiguousarray(ids, dtype=np.uint32).reshape(-1, 5)
        m = pts.shape[0]
        out = np.zeros(m, np.float32)
        ex = np.zeros(m, np.uint8)
        self.lib.orc_conflict_batch(U32(m), _ptr(pts), _ptr(ids), _ptr(out), _ptr(ex))
        return out, ex

    # ---- solver ----------------------------------------------------------------
    def cg_f32(self, row, col, val, b, x0, jacobi: bool = True):
        x = np.ascontiguousarray(x0, dtype=np.float32).copy()
        it = self.lib.orc_cg_f32(U32(len(row) - 1), _ptr(np.ascontiguousarray(row, np.uint32)),
                                 _ptr(np.ascontiguousarray(col, np.uint32)),
                                 _ptr(np.ascontiguousarray(val, np.float32)),
                                 _ptr(np.ascontiguousarray(b, np.float32)), _ptr(x),
                                 ctypes.c_int(int(jacobi)))
        return x, int(it)


class Reference:
    """The reference's own sources built for the host (``_ref``), if present."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.ref_ashape3d_run.restype = P
        self.lib.ref_cg_solve.restype = U32

    @staticmethod
    def available(path: str = REF_SO) -> bool:
        return os.path.exists(path)

    def lbvh3d(self, xyzr: np.ndarray) -> dict:
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        n = xyzr.shape[0]
        out = dict(
            bb_glob=np.zeros(6, np.float32), morton=np.zeros(n, np.uint64),
            perm=np.zeros(n, np.uint32), sep=np.zeros(n - 1, np.int32),
            cil=np.zeros(n - 1, np.uint8), leaf_parent=np.zeros(n, np.uint32),
            internal_parent=np.zeros(n - 1, np.uint32),
            bboxes=np.zeros((n - 1, 6), np.float32), obj_m=np.zeros((n, 4), np.float32))
        self.lib.ref_lbvh3d(U32(n), _ptr(xyzr),
                            *[_ptr(out[k]) for k in ("bb_glob", "morton", "perm", "sep", "cil",
                                                     "leaf_parent", "internal_parent", "bboxes",
                                                     "obj_m")])
        return out

    def trbvh3d(self, xyzr: np.ndarray, optimize: bool = False, threads: int | None = None) -> dict:
        """The reference's TRBVH: Apetrei build only, or the full build().

        Its SAH sums depend on which child reaches a node last
        (include/geometry/trbvh.hpp:371-373); threads=1 runs the leaves in
        index order, which makes them deterministic."""
        if threads is not None:
            gomp = ctypes.CDLL("libgomp.so.1")
            saved = gomp.omp_get_max_threads()
            gomp.omp_set_num_threads(int(threads))
            try:
                return self.trbvh3d(xyzr, optimize)
            finally:
                gomp.omp_set_num_threads(saved)
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        n = xyzr.shape[0]
        m = 2 * n - 1
        out = dict(child_left=np.zeros(n - 1, np.uint32), child_right=np.zeros(n - 1, np.uint32),
                   range_min=np.zeros(n - 1, np.uint32), range_max=np.zeros(n - 1, np.uint32),
                   parent=np.zeros(m, np.uint32), bboxes=np.zeros((m, 6), np.float32),
                   subtree_size=np.zeros(m, np.uint32), sah=np.zeros(m, np.float32), root=np.zeros(1, np.uint32),
                   obj_m=np.zeros((n, 4), np.float32))
        self.lib.ref_trbvh3d(U32(n), _ptr(xyzr), ctypes.c_int(int(optimize)),
                             *[_ptr(out[k]) for k in ("child_left", "child_right", "range_min", "range_max", "parent",
                                                      "bboxes", "subtree_size", "sah", "root", "obj_m")])
        out["root"] = int(out["root"][0])
        return out

    def lbvha3d(self, xyzr: np.ndarray) -> dict:
        """The reference's LBVHa (Apetrei agglomerative LBVH) over 3D spheres."""
        xyzr = np.ascontiguousarray(xyzr, dtype=np.float32)
        n = xyzr.shape[0]
        m = 2 * n - 1
        out = dict(children=np.zeros((n - 1, 2), np.uint32), range=np.zeros((n - 1, 2), np.uint32),
                   parent=np.zeros(m, np.uint32), bboxes=np.zeros((m, 6), np.float32), root=np.zeros(1, np.uint32),
                   obj_m=np.zeros((n, 4), np.float32))
        self.lib.ref_lbvha3d(U32(n), _ptr(xyzr), *[_ptr(out[k]) for k in ("children", "range", "parent", "bboxes",
                                                                         "root", "obj_m")])
        out["root"] = int(out["root"][0])
        return out

    def ashape3d(self, coords: np.ndarray, alpha: np.ndarray) -> AlphaShapeResult:
        coords = np.ascontiguousarray(coords, dtype=np.float32)
        alpha = np.ascontiguousarray(alpha, dtype=np.float32)
        n = coords.shape[0]
        h = self.lib.ref_ashape3d_run(U32(n), _ptr(coords), _ptr(alpha))
        try:
            nn, ne, ned = U32(), U32(), U32()
            self.lib.ref_ashape3d_sizes(P(h), ctypes.byref(nn), ctypes.byref(ne), ctypes.byref(ned))
            ne, ned = ne.value, ned.value
            r = AlphaShapeResult(
                perm=np.zeros(n, np.uint32), coords_m=np.zeros((n + 4, 4), np.float32),
                nineig=np.zeros(n, np.uint32), cand=np.zeros((n, 124), np.uint32),
                elems=np.zeros((ne, 4), np.uint32), row=np.zeros(n + 1, np.uint32),
                neig=np.zeros(ned, np.uint32), edge_is_bnd=np.zeros(ned, np.uint8),
                node_is_bnd=np.zeros(n, np.uint8), nelem=np.zeros(n, np.uint8))
            self.lib.ref_ashape3d_get(P(h), _ptr(r.perm), _ptr(r.elems), _ptr(r.row), _ptr(r.neig),
                                      _ptr(r.edge_is_bnd), _ptr(r.node_is_bnd), _ptr(r.nineig),
                                      _ptr(r.nelem), _ptr(r.coords_m))
            self.lib.ref_ashape3d_candidates(P(h), _ptr(r.cand))
        finally:
            self.lib.ref_ashape3d_free(P(h))
        return r

    def ashape2d(self, coords: np.ndarray, alpha: np.ndarray) -> AlphaShape2DResult:
        coords = np.ascontiguousarray(coords, dtype=np.float32).reshape(-1, 2)
        alpha = np.ascontiguousarray(alpha, dtype=np.float32)
        n = coords.shape[0]
        self.lib.ref_ashape2d_run.restype = P
        h = self.lib.ref_ashape2d_run(U32(n), _ptr(coords), _ptr(alpha))
        try:
            nn, ne, ned = U32(), U32(), U32()
            self.lib.ref_ashape2d_sizes(P(h), ctypes.byref(nn), ctypes.byref(ne), ctypes.byref(ned))
            ne, ned = ne.value, ned.value
            r = AlphaShape2DResult(
                perm=np.zeros(n, np.uint32), coords_m=np.zeros((n + 3, 3), np.float32),
                nineig=np.zeros(n, np.uint32), cand=np.zeros(0, np.uint32),
                elems=np.zeros((ne, 3), np.uint32), row=np.zeros(n + 1, np.uint32),
                neig=np.zeros(ned, np.uint32), edge_is_bnd=np.zeros(ned, np.uint8),
                node_is_bnd=np.zeros(n, np.uint8), nelem=np.zeros(n, np.uint8),
                bb_glob=np.zeros(4, np.float32), morton=np.zeros(n, np.uint64))
            self.lib.ref_ashape2d_get(P(h), _ptr(r.perm), _ptr(r.elems), _ptr(r.row), _ptr(r.neig),
                                      _ptr(r.edge_is_bnd), _ptr(r.node_is_bnd), _ptr(r.nineig),
                                      _ptr(r.nelem), _ptr(r.coords_m))
            self.lib.ref_ashape2d_lbvh(P(h), _ptr(r.bb_glob), _ptr(r.morton), None, None, None)
            w = int(max(1, int(r.nineig.max(initial=3)) - 3))
            r.cand = np.zeros((n, w), np.uint32)
            self.lib.ref_ashape2d_candidates(P(h), U32(w), _ptr(r.cand))
        finally:
            self.lib.ref_ashape2d_free(P(h))
        return r

    def mesh2d_order(self, xy: np.ndarray):
        """(perm[n], coords_m[n + 3, 2]) after the reference's Mesh2D_init
        (src/mesh/mesh.cpp:68-135): its Morton order and super nodes."""
        xy = np.ascontiguousarray(xy, dtype=np.float32).reshape(-1, 2)
        n = xy.shape[0]
        perm = np.zeros(n, np.uint32)
        coords_m = np.zeros((n + 3, 2), np.float32)
        self.lib.ref_mesh2d_order(U32(n), _ptr(xy), _ptr(perm), _ptr(coords_m))
        return perm, coords_m

    def cg_f32(self, row, col, val, b, x0, jacobi: bool = True):
        x = np.ascontiguousarray(x0, dtype=np.float32).copy()
        it = self.lib.ref_cg_solve(U32(len(row) - 1), _ptr(np.ascontiguousarray(row, np.uint32)),
                                   _ptr(np.ascontiguousarray(col, np.uint32)),
                                   _ptr(np.ascontiguousarray(val, np.float32)),
                                   _ptr(np.ascontiguousarray(b, np.float32)), _ptr(x),
                                   ctypes.c_int(int(jacobi)))
        return x, int(it)
