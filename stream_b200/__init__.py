"""stream_b200: B200-native PFEM remesh-and-solve path.

Drop-in for the reference's ``stream`` Python package on this path: the same
classes (``mesh.AlphaShape3D``, ``numerics.{HostCSR, DeviceCSR, LinSys,
PrecJacobi, SolverCG}``) over the same C ABI names, served by one CUDA library
built for sm_100a (``stream_b200/lib/libstream_b200.so``, with
``libmesh.so``/``libnumerics.so``/``libgeometry.so`` aliases).

There is no CPU fallback: importing the package fails if the library is
missing, and every compute call needs a B200 GPU.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(_HERE, "lib")
LIBPATH = os.path.join(LIBDIR, "libstream_b200.so")

if not os.path.exists(LIBPATH):
    raise ImportError(
        f"stream_b200: CUDA library not built ({LIBPATH} missing); run `python stream_b200/build.py`")

lib = ctypes.CDLL(LIBPATH)
# The reference loads three libraries (python/__init__.py:40-42); all three
# names resolve to the same binary here.
libgeo = libnum = libmesh = lib

# Status bits of include/stream_b200.h.
STREAM_ST_STACK_OVERFLOW = 0x001
STREAM_ST_WALK_CAP = 0x002
STREAM_ST_BROKEN_CYCLE = 0x004
STREAM_ST_TET_CAP = 0x008
STREAM_ST_EXACT_OVERFLOW = 0x010
STREAM_ST_LOOKBACK_TIMEOUT = 0x020
STREAM_ST_TRUNCATED = 0x040
STREAM_ST_BAD_INPUT = 0x080
STREAM_ST_CUDA_ERROR = 0x100

lib.stream_b200_last_error.restype = ctypes.c_char_p
lib.stream_b200_device_ok.restype = ctypes.c_int


def last_error() -> str:
    return lib.stream_b200_last_error().decode()


def device_ok() -> bool:
    """True when a B200 (compute capability 10.0) is visible."""
    return bool(lib.stream_b200_device_ok())


class StreamError(RuntimeError):
    """Raised when an additive (status-returning) entry point fails."""


def check(rc: int, what: str) -> None:
    if rc != 0:
        raise StreamError(f"{what} failed (status 0x{rc:x}): {last_error()}")


from . import geometry, mesh, numerics, pfem  # noqa: E402,F401
