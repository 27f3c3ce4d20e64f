"""Sparse linear algebra, same classes as the reference's ``stream.numerics``
(python/numerics/{csr,linsys,jacobi,cg}.py): HostCSR, DeviceCSR, LinSys,
PrecJacobi, SolverCG over the reference's C ABI names; plus the additive FP64 /
mixed-precision PoissonSystem."""
from __future__ import annotations

import ctypes

import numpy as np
import numpy.typing as npt

from .. import StreamError, check, last_error, libnum

_P = ctypes.c_void_p
_u32 = np.ctypeslib.ndpointer(dtype=np.uint32, ndim=1, flags=("C", "ALIGNED"))
_f32 = np.ctypeslib.ndpointer(dtype=np.float32, ndim=1, flags=("C", "ALIGNED"))
_f32w = np.ctypeslib.ndpointer(dtype=np.float32, ndim=1, flags=("C", "ALIGNED", "WRITEABLE"))

for _name, _res, _args in [
    ("d_csr_create", _P, []), ("d_csr_destroy", None, [_P]),
    ("h_csr_create", _P, [ctypes.c_uint32, _u32, _u32, _f32]), ("h_csr_destroy", None, [_P]),
    ("d_csr_h2d", None, [_P, _P]),
    ("LinSys_create", _P, []), ("LinSys_destroy", None, [_P]), ("LinSys_set", None, [_P, _P, _f32]),
    ("PrecJacobi_create", _P, [_P]), ("PrecJacobi_destroy", None, [_P]),
    ("SolverCG_create", _P, []), ("SolverCG_destroy", None, [_P]),
    ("SolverCG_jacobi_solve", ctypes.c_uint32, [_P, _P, _P, _f32w]),
    ("SolverCG_solve", ctypes.c_uint32, [_P, _P, _f32w]),
    ("PoissonSystem_create", _P, []), ("PoissonSystem_destroy", None, [_P]),
    ("PoissonSystem_assemble", ctypes.c_int, [_P, _P, ctypes.c_int, _P, ctypes.c_int]),
    ("PoissonSystem_set_csr", ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, _P, _P]),
    ("PoissonSystem_get_size", ctypes.c_int, [_P, _P, _P]),
    ("PoissonSystem_get_csr", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("PoissonSystem_solve", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_double, ctypes.c_uint32, ctypes.c_double,
                                           _P, _P]),
    ("PoissonSystem_get_solution", ctypes.c_int, [_P, _P]),
    ("PoissonSystem_assembly_stats", ctypes.c_int, [_P, _P]),
]:
    _fn = getattr(libnum, _name)
    _fn.restype = _res
    _fn.argtypes = _args


def _p(a):
    return a.ctypes.data_as(_P)


def _nonnull(h, what):
    if not h:
        raise StreamError(f"{what} failed: {last_error()}")
    return h


class HostCSR:
    def __init__(self, row: npt.NDArray[np.uint32], col: npt.NDArray[np.uint32], val: npt.NDArray[np.float32]):
        self.n = len(row) - 1
        self.nnz = int(row[self.n])
        self._keep = (np.ascontiguousarray(row, np.uint32), np.ascontiguousarray(col, np.uint32),
                      np.ascontiguousarray(val, np.float32))
        self.hcsr = _nonnull(libnum.h_csr_create(self.n, *self._keep), "h_csr_create")

    def __del__(self):
        if getattr(self, "hcsr", None):
            libnum.h_csr_destroy(self.hcsr)
            self.hcsr = None


class DeviceCSR:
    def __init__(self, host_csr: HostCSR):
        self.n = host_csr.n
        self.dcsr = _nonnull(libnum.d_csr_create(), "d_csr_create")
        self.set_from_host(host_csr)

    def __del__(self):
        if getattr(self, "dcsr", None):
            libnum.d_csr_destroy(self.dcsr)
            self.dcsr = None

    def set_from_host(self, host_csr: HostCSR):
        libnum.d_csr_h2d(self.dcsr, host_csr.hcsr)


class LinSys:
    def __init__(self, dcsr: DeviceCSR, b: npt.NDArray[np.float32]):
        self.sys = _nonnull(libnum.LinSys_create(), "LinSys_create")
        self.set(dcsr, b)

    def set(self, dcsr: DeviceCSR, b):
        libnum.LinSys_set(self.sys, dcsr.dcsr, np.ascontiguousarray(b, np.float32))

    def __del__(self):
        if getattr(self, "sys", None):
            libnum.LinSys_destroy(self.sys)
            self.sys = None


class PrecJacobi:
    def __init__(self, dcsr: DeviceCSR):
        self.prec = _nonnull(libnum.PrecJacobi_create(dcsr.dcsr), "PrecJacobi_create")

    def __del__(self):
        if getattr(self, "prec", None):
            libnum.PrecJacobi_destroy(self.prec)
            self.prec = None


class SolverCG:
    def __init__(self):
        self.solver = _nonnull(libnum.SolverCG_create(), "SolverCG_create")

    def __del__(self):
        if getattr(self, "solver", None):
            libnum.SolverCG_destroy(self.solver)
            self.solver = None

    def solve_jacobi(self, sys: LinSys, prec: PrecJacobi, x: npt.NDArray[np.float32]):
        if type(prec) is not PrecJacobi:
            raise TypeError(f"SolverCG.solve_jacobi expects a 'PrecJacobi' preconditioner, not a '{type(prec)}'")
        sol = np.copy(x).astype(np.float32)
        niter = libnum.SolverCG_jacobi_solve(self.solver, sys.sys, prec.prec, sol)
        x[:] = sol[:]
        return niter

    def solve(self, sys: LinSys, x: npt.NDArray[np.float32]):
        sol = np.copy(x).astype(np.float32)
        niter = libnum.SolverCG_solve(self.solver, sys.sys, sol)
        x[:] = sol[:]
        return niter


class PoissonSystem:
    """FP64 pressure system: P1 Laplacian assembled on the GPU from an
    AlphaShape3D, or a host FP64 CSR; solved by FP64 Jacobi-PCG (method 0) or
    mixed-precision iterative refinement (method 1)."""

    FP64_JACOBI = 0
    MIXED_IR = 1

    def __init__(self):
        self.h = _nonnull(libnum.PoissonSystem_create(), "PoissonSystem_create")

    def __del__(self):
        if getattr(self, "h", None):
            libnum.PoissonSystem_destroy(self.h)
            self.h = None

    def assemble(self, mesh, rhs: str = "one", modes: np.ndarray | None = None) -> None:
        kind = 0 if rhs == "one" else 1
        m = np.zeros((8, 5), np.float32) if modes is None else np.ascontiguousarray(modes, np.float32).reshape(-1, 5)
        check(libnum.PoissonSystem_assemble(self.h, mesh.mesh, kind, _p(m), len(m) if kind else 0), "assemble")

    def set_csr(self, row, col, val, b) -> None:
        row = np.ascontiguousarray(row, np.uint32)
        col = np.ascontiguousarray(col, np.uint32)
        val = np.ascontiguousarray(val, np.float64)
        b = np.ascontiguousarray(b, np.float64)
        check(libnum.PoissonSystem_set_csr(self.h, len(row) - 1, _p(row), _p(col), _p(val), _p(b)), "set_csr")

    def size(self):
        n, nnz = ctypes.c_uint32(), ctypes.c_uint32()
        check(libnum.PoissonSystem_get_size(self.h, ctypes.byref(n), ctypes.byref(nnz)), "get_size")
        return n.value, nnz.value

    def get_csr(self):
        n, nnz = self.size()
        row = np.empty(n + 1, np.uint32)
        col = np.empty(nnz, np.uint32)
        val = np.empty(nnz, np.float64)
        b = np.empty(n, np.float64)
        check(libnum.PoissonSystem_get_csr(self.h, _p(row), _p(col), _p(val), _p(b)), "get_csr")
        return row, col, val, b

    def solve(self, method: int = 0, rtol: float = 1e-8, maxit: int = 100000, inner_rtol: float = 1e-4,
              x0: np.ndarray | None = None):
        """Returns (x, report) with report keys iterations, outer, relres, ms, converged."""
        n, _ = self.size()
        x = np.zeros(n, np.float64) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        rep = np.zeros(6, np.float64)
        check(libnum.PoissonSystem_solve(self.h, method, rtol, maxit, inner_rtol, _p(x), _p(rep)), "solve")
        return x, dict(iterations=int(rep[0]), outer=int(rep[1]), relres=float(rep[2]), ms=float(rep[3]),
                       converged=bool(rep[4]))

    def isolated_rows(self) -> int:
        v = ctypes.c_uint32()
        check(libnum.PoissonSystem_assembly_stats(self.h, ctypes.byref(v)), "assembly_stats")
        return v.value
