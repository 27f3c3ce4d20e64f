"""Regenerate tests/golden/digests.json: per-array SHA-256 digests of the
oracle's outputs on full-size clouds (too large to commit as arrays).

Cases and the checker each one is pinned to:

* ``stress_4m`` -- the 4,000,000-point meshing-stress cloud (seed 0), alpha
  1.5 N^-1/3: LBVH arrays, TRBVH (treelet 7, 3D area) arrays and every
  mesher output from the plain-C restatement.  The reference build cannot run
  this cloud: it sizes its neighbour table by the uncapped neighbour counts
  (src/mesh/DirectAlphaShape3D.cpp:235-297), which for the blob cores overflow
  its 32-bit offsets.  The restatement equals the reference build bit for
  bit on every smaller cloud the tests run (uniform, lattice, blobs with
  truncated stars, duplicates, the sub-cube below).
* ``stress_subcube`` -- the 223,766 points of the 4M cloud in the corner box
  that the CPU baseline times (``workloads.sub_cube``, target 200,000):
  LBVH and mesher outputs of the reference build itself (oracle/_ref).
* ``uniform3d_*`` -- the reference's uniform3D cloud (glibc srand(42),
  testcases/IMR26/uniform3D.cpp:130-142): the published example (100,000
  points, alpha 0.022, testcases/IMR26/README.md:93-99) and the paper's sweep
  (README.md:80-86), from the reference build.

Usage: OMP_NUM_THREADS=<cores> python tests/golden/make_digests.py [case ...]
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
OUT = os.path.join(HERE, "digests.json")


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


dg = _load("_golden_digest", os.path.join(HERE, "digest.py"))
# pure-NumPy generators, loaded by path (no CUDA library needed)
wl = _load("_workloads", os.path.join(ROOT, "stream_b200", "workloads.py"))


def _xyzr(pts, al):
    return np.concatenate([pts, al[:, None]], 1).astype(np.float32)


def case_stress_4m():
    from oracle.oracle import Restatement
    R = Restatement()
    pts, al = wl.meshing_stress(4_000_000, seed=0)
    xyzr = _xyzr(pts, al)
    rec = {"generator": "workloads.meshing_stress(4_000_000, seed=0)", "checker": "restatement",
           "input": dg.input_digest(pts, al)}
    rec["lbvh"] = dg.tree_digests(R.lbvh3d(xyzr), dg.LBVH_KEYS)
    rec["trbvh_k7_3d"] = dg.tree_digests(R.trbvh3d(xyzr, treelet_size=7, area3d=True, rounds=3), dg.TRBVH_KEYS)
    r = R.ashape3d(pts, al)
    rec["mesh"] = dg.mesh_digests(dg.mesh_arrays_from_result(r))
    rec["mesh"]["n_truncated"] = int(r.n_truncated)
    return rec


def case_stress_subcube():
    from oracle.oracle import Reference
    F = Reference()
    pts4, al4 = wl.meshing_stress(4_000_000, seed=0)
    pts, al, s = wl.sub_cube(pts4, al4, 200_000)
    rec = {"generator": "workloads.sub_cube(*workloads.meshing_stress(4_000_000, seed=0), 200_000)",
           "checker": "reference", "points": int(len(pts)), "box_fraction": s, "input": dg.input_digest(pts, al)}
    rec["lbvh"] = dg.tree_digests(F.lbvh3d(_xyzr(pts, al)), dg.LBVH_KEYS)
    rec["mesh"] = dg.mesh_digests(dg.mesh_arrays_from_result(F.ashape3d(pts, al)))
    return rec


def case_uniform3d(n, alpha):
    from oracle.oracle import Reference
    F = Reference()
    pts, al = wl.glibc_uniform_cube(n, alpha)
    rec = {"generator": f"workloads.glibc_uniform_cube({n}, {alpha})", "checker": "reference",
           "points": n, "alpha": alpha, "input": dg.input_digest(pts, al)}
    rec["mesh"] = dg.mesh_digests(dg.mesh_arrays_from_result(F.ashape3d(pts, al)))
    return rec


def cases():
    yield "uniform3d_100000_0.022", lambda: case_uniform3d(100_000, 0.022)
    for n, a in wl.UNIFORM3D_SWEEP:
        yield f"uniform3d_{n}_{a}", (lambda n=n, a=a: case_uniform3d(n, a))
    yield "stress_subcube", case_stress_subcube
    yield "stress_4m", case_stress_4m


def main(argv):
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    for name, fn in cases():
        if argv and name not in argv:
            continue
        t0 = time.time()
        data[name] = fn()
        m = data[name].get("mesh", {})
        print(f"{name}: {m.get('n_elems')} tets, {time.time() - t0:.1f} s", flush=True)
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:])
