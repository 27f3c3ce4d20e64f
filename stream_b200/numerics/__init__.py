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
    ("PrecJacobi_get_status", ctypes.c_int, [_P, _P]),
    ("SolverCG_get_termination", ctypes.c_int, [_P]),
    ("PoissonSystem_create", _P, []), ("PoissonSystem_destroy", None, [_P]),
    ("PoissonSystem_assemble", ctypes.c_int, [_P, _P, ctypes.c_int, _P, ctypes.c_int]),
    ("PoissonSystem_set_csr", ctypes.c_int, [_P, ctypes.c_uint32, _P, _P, _P, _P]),
    ("PoissonSystem_get_size", ctypes.c_int, [_P, _P, _P]),
    ("PoissonSystem_get_csr", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("PoissonSystem_solve", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_double, ctypes.c_uint32, ctypes.c_double,
                                           _P, _P]),
    ("PoissonSystem_get_solution", ctypes.c_int, [_P, _P]),
    ("PoissonSystem_assembly_stats", ctypes.c_int, [_P, _P]),
    ("PoissonSystem_set_coords", ctypes.c_int, [_P, _P]),
    ("PoissonSystem_set_fsai", ctypes.c_int, [_P, _P]),
    ("PoissonSystem_get_fsai", ctypes.c_int, [_P, _P, _P, _P]),
    ("PoissonSystem_fsai_stats", ctypes.c_int, [_P, _P]),
    ("PoissonSystem_get_ky", ctypes.c_int, [_P, _P, _P]),
    ("FsaiModel_param_count", ctypes.c_uint32, []),
    ("FsaiModel_create", _P, []), ("FsaiModel_destroy", None, [_P]),
    ("FsaiModel_set_params", ctypes.c_int, [_P, _P, ctypes.c_uint32]),
    ("FsaiModel_get_params", ctypes.c_int, [_P, _P, ctypes.c_uint32]),
    ("FsaiModel_reset_optimizer", ctypes.c_int, [_P]),
    ("FsaiModel_set_loss", ctypes.c_int, [_P, ctypes.c_uint32]),
    ("FsaiModel_set_base", ctypes.c_int, [_P, ctypes.c_uint32]),
    ("FsaiModel_get_base", ctypes.c_int, [_P, _P]),
    ("FsaiModel_loss_grad", ctypes.c_int, [_P, _P, ctypes.c_uint64, _P, _P, _P]),
    ("FsaiModel_train_step", ctypes.c_int, [_P, _P, ctypes.c_uint64, ctypes.c_float, ctypes.c_float, _P]),
    ("FsaiModel_train_batch", ctypes.c_int, [_P, _P, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_float,
                                             ctypes.c_float, _P]),
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

    def __del__(self, _destroy=libnum.h_csr_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "hcsr", None):
            _destroy(self.hcsr)
            self.hcsr = None


class DeviceCSR:
    def __init__(self, host_csr: HostCSR):
        self.n = host_csr.n
        self.dcsr = _nonnull(libnum.d_csr_create(), "d_csr_create")
        self.set_from_host(host_csr)

    def __del__(self, _destroy=libnum.d_csr_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "dcsr", None):
            _destroy(self.dcsr)
            self.dcsr = None

    def set_from_host(self, host_csr: HostCSR):
        libnum.d_csr_h2d(self.dcsr, host_csr.hcsr)


class LinSys:
    def __init__(self, dcsr: DeviceCSR, b: npt.NDArray[np.float32]):
        self.sys = _nonnull(libnum.LinSys_create(), "LinSys_create")
        self.set(dcsr, b)

    def set(self, dcsr: DeviceCSR, b):
        libnum.LinSys_set(self.sys, dcsr.dcsr, np.ascontiguousarray(b, np.float32))

    def __del__(self, _destroy=libnum.LinSys_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "sys", None):
            _destroy(self.sys)
            self.sys = None


class PrecJacobi:
    def __init__(self, dcsr: DeviceCSR):
        self.prec = _nonnull(libnum.PrecJacobi_create(dcsr.dcsr), "PrecJacobi_create")

    def bad_rows(self) -> int:
        """Rows whose diagonal entry is missing, zero or has no finite inverse
        (additive; the reference would use an uninitialised inverse there)."""
        v = ctypes.c_uint32()
        libnum.PrecJacobi_get_status(self.prec, ctypes.byref(v))
        return v.value

    def __del__(self, _destroy=libnum.PrecJacobi_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "prec", None):
            _destroy(self.prec)
            self.prec = None


class SolverCG:
    def __init__(self):
        self.solver = _nonnull(libnum.SolverCG_create(), "SolverCG_create")

    def __del__(self, _destroy=libnum.SolverCG_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "solver", None):
            _destroy(self.solver)
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

    TERMINATION = {0: "none", 1: "converged", 2: "iteration_cap", 3: "breakdown"}

    def termination(self) -> str:
        """How the last solve ended (additive): converged (the reference's
        stopping rule), iteration_cap, breakdown (non-finite r.z) or none."""
        return self.TERMINATION[int(libnum.SolverCG_get_termination(self.solver))]


class PoissonSystem:
    """FP64 pressure system: P1 Laplacian assembled on the GPU from an
    AlphaShape3D, or a host FP64 CSR; solved by FP64 Jacobi-PCG (method 0),
    mixed-precision iterative refinement with Jacobi (method 1) or with the
    learned FSAI preconditioner of an attached FsaiModel (method 2)."""

    FP64_JACOBI = 0
    MIXED_IR = 1
    FSAI_MIXED = 2
    KY_FSAI_MIXED = 3  # the Kolotilina-Yeremin FSAI (exact local solves) in the same refinement

    def __init__(self):
        self.h = _nonnull(libnum.PoissonSystem_create(), "PoissonSystem_create")

    def __del__(self, _destroy=libnum.PoissonSystem_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "h", None):
            _destroy(self.h)
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

    def solve(self, method: int = 0, rtol: float = 1e-8, maxit: int = 100000, inner_rtol: float = 0.0,
              x0: np.ndarray | None = None):
        """Returns (x, report) with report keys iterations, outer, relres, ms,
        converged, fallback."""
        n, _ = self.size()
        x = np.zeros(n, np.float64) if x0 is None else np.ascontiguousarray(x0, np.float64).copy()
        rep = np.zeros(6, np.float64)
        check(libnum.PoissonSystem_solve(self.h, method, rtol, maxit, inner_rtol, _p(x), _p(rep)), "solve")
        return x, dict(iterations=int(rep[0]), outer=int(rep[1]), relres=float(rep[2]), ms=float(rep[3]),
                       converged=bool(rep[4]), fallback=bool(rep[5]))

    def set_coords(self, xyz) -> None:
        xyz = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        check(libnum.PoissonSystem_set_coords(self.h, _p(xyz)), "set_coords")

    def set_fsai(self, model: "FsaiModel | None") -> None:
        self._model = model  # the system uses the model until detached
        check(libnum.PoissonSystem_set_fsai(self.h, model.h if model is not None else None), "set_fsai")

    def fsai_g(self) -> np.ndarray:
        """G of the attached model aligned with the CSR (lower: G_ij, upper: G_ji)."""
        _, nnz = self.size()
        g = np.empty(nnz, np.float32)
        check(libnum.PoissonSystem_get_fsai(self.h, _p(g), None, None), "get_fsai")
        return g

    def fsai_features(self) -> np.ndarray:
        ne = ctypes.c_uint32()
        check(libnum.PoissonSystem_get_fsai(self.h, None, None, ctypes.byref(ne)), "get_fsai")
        f = np.empty((ne.value, 16), np.float32)
        check(libnum.PoissonSystem_get_fsai(self.h, None, _p(f), None), "get_fsai")
        return f

    def fsai_stats(self) -> dict:
        st = np.zeros(4, np.float64)
        check(libnum.PoissonSystem_fsai_stats(self.h, _p(st)), "fsai_stats")
        return dict(setup_ms=float(st[0]), infer_ms=float(st[1]), fallback=bool(st[2]), lower_edges=int(st[3]))

    def ky_g(self):
        """(G, rows left diagonal) of the Kolotilina-Yeremin FSAI (method 3),
        G aligned with the CSR like fsai_g()."""
        _, nnz = self.size()
        g = np.empty(nnz, np.float32)
        rows = ctypes.c_uint32()
        check(libnum.PoissonSystem_get_ky(self.h, _p(g), ctypes.byref(rows)), "get_ky")
        return g, rows.value

    def isolated_rows(self) -> int:
        v = ctypes.c_uint32()
        check(libnum.PoissonSystem_assembly_stats(self.h, ctypes.byref(v)), "assembly_stats")
        return v.value


class FsaiModel:
    """Parameters and Adam state of the learned FSAI network (on the GPU)."""

    PARAM_COUNT = 9473
    LOSSES = {"residual": 0, "kaporin": 1}
    BASES = {"none": 0, "ky": 1}

    def __init__(self, params: np.ndarray | None = None, loss: str = "residual", base: str = "none"):
        assert libnum.FsaiModel_param_count() == self.PARAM_COUNT
        self.h = _nonnull(libnum.FsaiModel_create(), "FsaiModel_create")
        if params is not None:
            self.set_params(params)
        self.set_loss(loss)
        self.set_base(base)

    def set_base(self, base: str) -> None:
        """What the output corrects: "none" (zero output = Jacobi) or "ky", the
        Kolotilina-Yeremin G of the system (zero output = that G; its value is
        input feature 10)."""
        if base not in self.BASES:
            raise ValueError(f"unknown FSAI base {base!r}; expected one of {sorted(self.BASES)}")
        check(libnum.FsaiModel_set_base(self.h, self.BASES[base]), "FsaiModel_set_base")
        self.base = base

    def set_loss(self, loss: str) -> None:
        """Training loss: "residual" sum_p ||G A G^T z_p - z_p||^2 / (16 n), or
        "kaporin" log(t/n) - (2/n) sum_i log G_ii, t = sum_p z_p^T G A G^T z_p / 16."""
        if loss not in self.LOSSES:
            raise ValueError(f"unknown FSAI loss {loss!r}; expected one of {sorted(self.LOSSES)}")
        check(libnum.FsaiModel_set_loss(self.h, self.LOSSES[loss]), "FsaiModel_set_loss")
        self.loss = loss

    def __del__(self, _destroy=libnum.FsaiModel_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "h", None):
            _destroy(self.h)
            self.h = None

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32).reshape(-1)
        check(libnum.FsaiModel_set_params(self.h, _p(p), len(p)), "FsaiModel_set_params")

    def get_params(self) -> np.ndarray:
        p = np.empty(self.PARAM_COUNT, np.float32)
        check(libnum.FsaiModel_get_params(self.h, _p(p), len(p)), "FsaiModel_get_params")
        return p

    def reset_optimizer(self) -> None:
        check(libnum.FsaiModel_reset_optimizer(self.h), "FsaiModel_reset_optimizer")

    def loss_grad(self, ps: PoissonSystem, seed: int = 0, probes: np.ndarray | None = None):
        """(loss, gradient) of the model's training loss over 16 probes."""
        g = np.empty(self.PARAM_COUNT, np.float32)
        loss = ctypes.c_double()
        z = None if probes is None else np.ascontiguousarray(probes, np.float32)
        check(libnum.FsaiModel_loss_grad(self.h, ps.h, seed, _p(z) if z is not None else None, ctypes.byref(loss),
                                         _p(g)), "FsaiModel_loss_grad")
        return loss.value, g

    def train_step(self, ps: PoissonSystem, seed: int, lr: float, clip: float = 0.0) -> float:
        loss = ctypes.c_double()
        check(libnum.FsaiModel_train_step(self.h, ps.h, seed, lr, clip, ctypes.byref(loss)), "FsaiModel_train_step")
        return loss.value

    def train_batch(self, systems, seed: int, lr: float, clip: float = 0.0) -> float:
        """One Adam step on the mean loss of several systems."""
        hs = (ctypes.c_void_p * len(systems))(*[ps.h for ps in systems])
        loss = ctypes.c_double()
        check(libnum.FsaiModel_train_batch(self.h, hs, len(systems), seed, lr, clip, ctypes.byref(loss)),
              "FsaiModel_train_batch")
        return loss.value

    @staticmethod
    def weights_path(base: str = "none") -> str:
        import os
        name = "fsai_weights.npy" if base == "none" else f"fsai_weights_{base}.npy"
        return os.path.join(os.path.dirname(os.path.dirname(__file__)), name)

    @classmethod
    def trained(cls, base: str = "none") -> "FsaiModel":
        """A network trained by stream_b200.fsai_train: base "none" (corrects
        Jacobi; shipped with the package) or "ky" (corrects the
        Kolotilina-Yeremin G; written by fsai_train --base ky, not shipped)."""
        return cls(np.load(cls.weights_path(base)), base=base)
