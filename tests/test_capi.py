"""CPU: the C-ABI library builds, loads and exports every symbol that
include/stream_b200.h declares (no compute calls without a GPU)."""
import ctypes
import os
import re
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "stream_b200.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", src)
    return sorted(set(names))


def test_header_declares_reference_names():
    d = set(_declared())
    for name in ("AlphaShape3D_create", "AlphaShape3D_destroy", "AlphaShape3D_set_nodes", "AlphaShape3D_init",
                 "AlphaShape3D_compute", "AlphaShape3D_get_nelem", "AlphaShape3D_get_elem",
                 "AlphaShape3D_get_ordered_nodes", "d_csr_create", "d_csr_destroy", "h_csr_create",
                 "h_csr_destroy", "d_csr_h2d", "LinSys_create", "LinSys_destroy", "LinSys_set",
                 "PrecJacobi_create", "PrecJacobi_destroy", "SolverCG_create", "SolverCG_destroy",
                 "SolverCG_jacobi_solve", "SolverCG_solve",
                 # src/mesh/DirectAlphaShape2D.cpp:698-753
                 "AlphaShape2D_create", "AlphaShape2D_destroy", "AlphaShape2D_set_nodes", "AlphaShape2D_init",
                 "AlphaShape2D_compute", "AlphaShape2D_get_nelem", "AlphaShape2D_get_elem",
                 "AlphaShape2D_get_ordered_nodes",
                 # src/mesh/mesh.cpp:806-862
                 "Mesh2D_create", "Mesh2D_destroy", "Mesh2D_set_nodes", "Mesh2D_init",
                 "Mesh2D_insert_morton_neighbors", "Mesh2D_insert_BVH_neighbors", "Mesh2D_insert_iterative",
                 "Mesh2D_remove_super_nodes", "Mesh2D_get_nelem", "Mesh2D_get_elem", "Mesh2D_get_ordered_nodes"):
        assert name in d, name


def test_library_exports_every_declared_symbol():
    from stream_b200 import build
    lib = build.build()
    handle = ctypes.CDLL(lib)
    missing = [n for n in _declared() if not hasattr(handle, n)]
    assert not missing, missing


def test_reference_library_names_resolve():
    from stream_b200 import build
    build.build()
    for alias in ("libmesh.so", "libnumerics.so", "libgeometry.so"):
        p = os.path.join(ROOT, "stream_b200", "lib", alias)
        assert os.path.exists(p)
        assert hasattr(ctypes.CDLL(p), "AlphaShape3D_create")


def test_only_c_abi_is_exported():
    from stream_b200 import build
    lib = build.build()
    out = subprocess.run(["nm", "-D", "--defined-only", lib], capture_output=True, text=True).stdout
    syms = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert syms <= set(_declared()) | {"_init", "_fini"}, sorted(syms - set(_declared()))


def test_header_compiles_as_c():
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", HEADER],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_package_imports_without_gpu():
    import stream_b200
    assert stream_b200.device_ok() in (True, False)


def _header_status_bits():
    src = open(HEADER).read()
    return {name: int(v, 16) for name, v in re.findall(r"#define STREAM_ST_([A-Z_]+)\s+(0x[0-9a-fA-F]+)", src)}


def test_python_status_tables_match_the_header():
    """The Python mesh classes decode status words with the header's bits
    (the 2D mesher reports its triangle-list overflow on the TET_CAP bit)."""
    from stream_b200.mesh import ashape2d, ashape3d, mesh2d
    bits = _header_status_bits()
    names3 = {"stack_overflow": "STACK_OVERFLOW", "walk_cap": "WALK_CAP", "broken_cycle": "BROKEN_CYCLE",
              "tet_cap": "TET_CAP", "exact_overflow": "EXACT_OVERFLOW", "lookback_timeout": "LOOKBACK_TIMEOUT",
              "truncated": "TRUNCATED", "bad_input": "BAD_INPUT", "cuda_error": "CUDA_ERROR"}
    for bit, name in ashape3d.STATUS_BITS.items():
        assert bits[names3[name]] == bit, name
    names2 = dict(names3, tri_cap="TET_CAP")
    for bit, name in ashape2d.STATUS_BITS.items():
        assert bits[names2[name]] == bit, name
    names_m = dict(names3, query_budget="WALK_CAP", local_id_cap="TET_CAP", incomplete="INCOMPLETE")
    for bit, name in mesh2d.STATUS_BITS.items():
        assert bits[names_m[name]] == bit, name
    for mod in (ashape2d, ashape3d, mesh2d):
        assert mod.ERROR_BITS & bits["CUDA_ERROR"] and mod.ERROR_BITS & bits["BAD_INPUT"]
        assert not mod.ERROR_BITS & bits["TRUNCATED"]


# Modules of the reference's Python package whose bindings this library serves
# (tests/golden/reference_bindings.json, made from the reference's python/
# sources by tests/golden/make_bindings.py).
SERVED = ("python/mesh/ashape2D.py", "python/mesh/ashape3D.py", "python/mesh/mesh.py", "python/numerics/cg.py",
          "python/numerics/csr.py", "python/numerics/jacobi.py", "python/numerics/linsys.py")


def test_reference_python_bindings_resolve():
    """Every C entry point that the reference's ashape2D, ashape3D, mesh, csr,
    linsys, jacobi and cg modules bind at import time is exported by this library."""
    import json
    from stream_b200 import build
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "reference_bindings.json")))
    handle = ctypes.CDLL(build.build())
    for mod in SERVED:
        missing = [n for n in want[mod] if not hasattr(handle, n)]
        assert not missing, (mod, missing)
    assert set(want) == set(SERVED)


def test_reference_python_modules_import_against_this_library():
    """The reference's own binding modules, unmodified, executed against this
    library (libmesh / libnumerics / libgeometry resolve to it): each module's
    import-time ctypes bindings succeed and its classes are defined.  Needs the
    reference tree (STREAM_REFERENCE)."""
    import importlib.util
    import sys
    import types

    import pytest
    ref = os.environ.get("STREAM_REFERENCE")
    if not ref or not os.path.isdir(os.path.join(ref, "python")):
        pytest.skip("STREAM_REFERENCE does not name the reference tree")
    from stream_b200 import build
    lib = ctypes.CDLL(build.build())
    pkg = types.ModuleType("_refstream")
    pkg.__path__ = []
    pkg.libgeo = pkg.libnum = pkg.libmesh = lib
    sys.modules["_refstream"] = pkg
    try:
        for sub in ("mesh", "numerics"):
            sp = types.ModuleType(f"_refstream.{sub}")
            sp.__path__ = [os.path.join(ref, "python", sub)]
            sys.modules[f"_refstream.{sub}"] = sp
        classes = {"python/mesh/ashape2D.py": "AlphaShape2D", "python/mesh/ashape3D.py": "AlphaShape3D",
                   "python/mesh/mesh.py": "Mesh2D",
                   "python/numerics/csr.py": "DeviceCSR", "python/numerics/linsys.py": "LinSys",
                   "python/numerics/jacobi.py": "PrecJacobi", "python/numerics/cg.py": "SolverCG"}
        for mod in ("python/numerics/csr.py", "python/numerics/linsys.py", "python/numerics/jacobi.py",
                    "python/numerics/cg.py", "python/mesh/ashape2D.py", "python/mesh/ashape3D.py",
                    "python/mesh/mesh.py"):
            sub, name = mod.split("/")[1], os.path.basename(mod)[:-3]
            full = f"_refstream.{sub}.{name}"
            spec = importlib.util.spec_from_file_location(full, os.path.join(ref, mod))
            m = importlib.util.module_from_spec(spec)
            sys.modules[full] = m
            spec.loader.exec_module(m)
            assert hasattr(m, classes[mod]), mod
    finally:
        for k in [k for k in sys.modules if k.startswith("_refstream")]:
            del sys.modules[k]
