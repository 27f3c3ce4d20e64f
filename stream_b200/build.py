"""Build the stream_b200 CUDA library in-tree for sm_100a.

Produces ``stream_b200/lib/libstream_b200.so`` (all kernels and the C ABI of
``include/stream_b200.h``) plus ``libmesh.so``, ``libnumerics.so`` and
``libgeometry.so`` symlinks, the library names the reference's ctypes package
loads (python/__init__.py:40-42 in the reference), so either front end can
bind the same binary.

Usage: ``python stream_b200/build.py [--force] [--jobs N]`` (by path: importing the package
would bind the library being built).
"""
from __future__ import annotations

import argparse
import hashlib
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIBNAME = "libstream_b200.so"
ALIASES = ("libmesh.so", "libnumerics.so", "libgeometry.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
BASE = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC,-fvisibility=hidden,-O2", "-Xptxas", "-warn-spills"]
# Files whose float arithmetic must match the reference operation by operation
# (no multiply-add contraction; explicit fmaf() calls stay fused).
NO_FMAD = {"ashape3d.cu", "ashape2d.cu", "mesh2d.cu", "lbvh.cu", "trbvh.cu", "predicates_noalloc.cu"}
SOURCES = ["capi_common.cu", "radix_sort.cu", "scan.cu", "lbvh.cu", "trbvh.cu", "ashape3d.cu", "capi_mesh.cu", "ashape2d.cu", "capi_mesh2d.cu", "mesh2d.cu", "capi_delaunay2d.cu",
           "numerics.cu", "fsai.cu", "capi_numerics.cu", "pfem.cu", "pfem_fs.cu", "capi_pfem.cu", "predicates_noalloc.cu"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the stream_b200 CUDA library cannot be built")


def _digest(paths) -> str:
    h = hashlib.sha256()
    for p in sorted(paths):
        with open(p, "rb") as f:
            h.update(p.encode())
            h.update(f.read())
    h.update(" ".join(ARCH + BASE + sorted(NO_FMAD)).encode())
    return h.hexdigest()


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    """Compile (if sources changed) and return the library path."""
    nvcc = _nvcc()
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    inc = os.path.join(os.path.dirname(HERE), "include")
    headers += [os.path.join(inc, f) for f in os.listdir(inc) if f.endswith(".h")]
    digest = _digest(srcs + headers)
    lib = os.path.join(LIBDIR, LIBNAME)
    stamp = os.path.join(LIBDIR, ".build_digest")
    if not force and os.path.exists(lib) and os.path.exists(stamp):
        with open(stamp) as f:
            if f.read().strip() == digest:
                return lib
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)

    def compile_one(src: str) -> str:
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        flags = list(BASE)
        if os.path.basename(src) in NO_FMAD:
            flags.append("-fmad=false")
        cmd = [nvcc, *ARCH, *flags, "-I", CSRC, "-I", inc, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr.strip():
            print(r.stderr, flush=True)
        return obj

    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = lib + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-Xcompiler", "-fPIC"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    for alias in ALIASES:
        p = os.path.join(LIBDIR, alias)
        if os.path.lexists(p):
            os.remove(p)
        os.symlink(LIBNAME, p)
    with open(stamp, "w") as f:
        f.write(digest)
    return lib


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args(argv)
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))
    return 0


if __name__ == "__main__":
    sys.exit(main())
