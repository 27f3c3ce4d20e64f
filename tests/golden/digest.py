"""SHA-256 digests of mesher, LBVH and TRBVH outputs (test infrastructure).

Full-size outputs (the 4M-point meshing-stress cloud gives 37.8M tets and a
2 GB candidate table) are too large to commit, so their fixtures hold one
digest per array.  Each array is hashed in a canonical form: C order, the
dtype the reference uses, little-endian bytes.  Candidate slots past a star's
size are zeroed first (their content is unspecified on both sides).
"""
from __future__ import annotations

import hashlib

import numpy as np

MESH_KEYS = ("perm", "nodes", "nineig", "cand", "nelem", "node_is_bnd", "row", "neig", "edge_is_bnd", "elems")
LBVH_KEYS = ("bb_glob", "morton", "perm", "sep", "cil", "leaf_parent", "internal_parent", "bboxes", "obj_m")
TRBVH_KEYS = ("child_left", "child_right", "range_min", "range_max", "parent", "bboxes", "subtree_size", "sah",
              "root", "obj_m")
DTYPES = {"perm": np.uint32, "nodes": np.float32, "nineig": np.uint32, "cand": np.uint32, "nelem": np.uint8,
          "node_is_bnd": np.uint8, "row": np.uint32, "neig": np.uint32, "edge_is_bnd": np.uint8,
          "elems": np.uint32, "bb_glob": np.float32, "morton": np.uint64, "sep": np.int32, "cil": np.uint8,
          "leaf_parent": np.uint32, "internal_parent": np.uint32, "bboxes": np.float32, "obj_m": np.float32,
          "child_left": np.uint32, "child_right": np.uint32, "range_min": np.uint32, "range_max": np.uint32,
          "parent": np.uint32, "subtree_size": np.uint32, "sah": np.float32, "root": np.uint32,
          "pts": np.float32, "alpha": np.float32}


def sha(a, dtype=None) -> str:
    a = np.ascontiguousarray(np.asarray(a, dtype=dtype) if dtype is not None else np.asarray(a))
    h = hashlib.sha256()
    h.update(str(a.shape).encode())
    h.update(a.astype(a.dtype.newbyteorder("<"), copy=False).tobytes())
    return h.hexdigest()


def mesh_arrays_from_result(r) -> dict:
    """Arrays of an oracle AlphaShapeResult (restatement or reference build)."""
    n = len(r.perm)
    return dict(perm=r.perm, nodes=r.coords_m[:n, :3], nineig=r.nineig, cand=r.cand, nelem=r.nelem,
                node_is_bnd=r.node_is_bnd, row=r.row, neig=r.neig, edge_is_bnd=r.edge_is_bnd, elems=r.elems)


def mesh_digests(arrs: dict) -> dict:
    """Digests of the mesher outputs; arrs holds MESH_KEYS."""
    out = {}
    nineig = np.asarray(arrs["nineig"]).astype(np.int64)
    for k in MESH_KEYS:
        a = arrs[k]
        if k == "cand":
            a = np.asarray(a, np.uint32).reshape(len(nineig), 124).copy()
            a[np.arange(124)[None, :] >= (nineig[:, None] - 4)] = 0
        out[k] = sha(a, DTYPES[k])
    out["n_elems"] = int(len(arrs["elems"]))
    out["n_edges"] = int(len(arrs["neig"]))
    return out


def tree_digests(arrs: dict, keys) -> dict:
    return {k: sha(np.atleast_1d(np.asarray(arrs[k])), DTYPES[k]) for k in keys}


def input_digest(pts, alpha) -> str:
    return sha(np.concatenate([np.asarray(pts, np.float32).reshape(len(alpha), -1),
                               np.asarray(alpha, np.float32)[:, None]], 1), np.float32)
