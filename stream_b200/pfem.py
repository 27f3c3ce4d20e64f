"""PFEM step loop on the GPU: Taylor-Green advection of the particles, or the
fractional-step flow solver (gravity, viscosity, box walls: Physics), remesh
(LBVH + alpha-shape Delaunay, free surface), P1 pressure assembly and the
learned-FSAI mixed-precision solve (Jacobi-PCG fallback) every step, over the
C ABI of include/stream_b200.h (PfemLoop_*).  The reference has no step loop;
its mesher and solver are the pieces this loop drives."""
from __future__ import annotations

import ctypes
import math

import numpy as np

from . import StreamError, check, lib
from .numerics import FsaiModel, _nonnull, _p

_P = ctypes.c_void_p
for _name, _res, _args in [
    ("stream_b200_advect_taylor_green", ctypes.c_int, [ctypes.c_uint32, _P, _P, ctypes.c_double, ctypes.c_uint32]),
    ("PfemLoop_create", _P, []), ("PfemLoop_destroy", None, [_P]),
    ("PfemLoop_set_particles", ctypes.c_int, [_P, ctypes.c_uint32, _P, ctypes.c_float]),
    ("PfemLoop_get_particles", ctypes.c_int, [_P, _P]),
    ("PfemLoop_set_flow", ctypes.c_int, [_P, _P]),
    ("PfemLoop_set_rhs_modes", ctypes.c_int, [_P, _P, ctypes.c_int]),
    ("PfemLoop_set_fsai", ctypes.c_int, [_P, _P]),
    ("PfemLoop_step", ctypes.c_int, [_P, ctypes.c_double, ctypes.c_double, _P]),
    ("PfemLoop_get_pressure", ctypes.c_int, [_P, _P]),
    ("PfemLoop_set_pressure", ctypes.c_int, [_P, _P]),
    ("PfemLoop_stats", ctypes.c_int, [_P, _P]),
    ("PfemLoop_set_physics", ctypes.c_int, [_P, _P]),
    ("PfemLoop_get_velocity", ctypes.c_int, [_P, _P]),
    ("PfemLoop_set_velocity", ctypes.c_int, [_P, _P]),
]:
    _fn = getattr(lib, _name)
    _fn.restype = _res
    _fn.argtypes = _args


class TaylorGreen:
    """u = amp R^T (sin kx' cos ky' cos kz', -cos kx' sin ky' cos kz', 0), x' = R (x - c)."""

    def __init__(self, rot=None, center=(0.0, 0.0, 0.0), k=2 * math.pi, amp=0.5):
        self.rot = np.eye(3) if rot is None else np.asarray(rot, np.float64).reshape(3, 3)
        self.center = np.asarray(center, np.float64).reshape(3)
        self.k = float(k)
        self.amp = float(amp)

    def packed(self) -> np.ndarray:
        return np.concatenate([self.rot.reshape(-1), self.center, [self.k, self.amp]]).astype(np.float64)

    def velocity(self, x: np.ndarray) -> np.ndarray:
        xp = (np.asarray(x, np.float64) - self.center) @ self.rot.T
        kx, ky, kz = self.k * xp[:, 0], self.k * xp[:, 1], self.k * xp[:, 2]
        up = np.stack([np.sin(kx) * np.cos(ky) * np.cos(kz), -np.cos(kx) * np.sin(ky) * np.cos(kz),
                       np.zeros(len(xp))], 1) * self.amp
        return up @ self.rot

    @classmethod
    def random(cls, rng, amp=None):
        rot, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        return cls(rot, rng.uniform(0.0, 0.8, 3), 2 * math.pi / rng.uniform(0.2, 0.8),
                   rng.uniform(0.2, 1.0) if amp is None else amp)


class Physics:
    """Fractional-step dynamics of the particles: gravity g, kinematic
    viscosity nu, density rho, in the box lo..hi (walls on all six faces)."""

    def __init__(self, g=(0.0, -9.81, 0.0), nu=1e-6, rho=1000.0, lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
        self.g = np.asarray(g, np.float64).reshape(3)
        self.nu, self.rho = float(nu), float(rho)
        self.lo = np.asarray(lo, np.float64).reshape(3)
        self.hi = np.asarray(hi, np.float64).reshape(3)

    def packed(self) -> np.ndarray:
        return np.concatenate([self.g, [self.nu, self.rho], self.lo, self.hi]).astype(np.float64)


def advect_taylor_green(xyz: np.ndarray, flow: TaylorGreen, dt: float, steps: int) -> np.ndarray:
    """Euler steps of the field on the GPU; returns the new FP64 positions."""
    x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3).copy()
    check(lib.stream_b200_advect_taylor_green(len(x), _p(x), _p(flow.packed()), dt, steps), "advect_taylor_green")
    return x


REPORT_KEYS = ("advect_ms", "remesh_ms", "assembly_ms", "precond_ms", "solve_ms", "step_ms", "iterations",
               "fallback", "nodes", "tets", "relres", "converged")


class PfemLoop:
    def __init__(self, xyz: np.ndarray, alpha: float, flow: TaylorGreen | None = None,
                 rhs_modes: np.ndarray | None = None, model: FsaiModel | None = None):
        self.h = _nonnull(lib.PfemLoop_create(), "PfemLoop_create")
        self.set_particles(xyz, alpha)
        self.set_flow(flow or TaylorGreen())
        if rhs_modes is not None:
            m = np.ascontiguousarray(rhs_modes, np.float32).reshape(-1, 5)
            self._modes = m
            check(lib.PfemLoop_set_rhs_modes(self.h, _p(m), len(m)), "PfemLoop_set_rhs_modes")
        self.set_fsai(model)

    def __del__(self, _destroy=lib.PfemLoop_destroy):  # bound at definition: module globals are gone at exit
        if getattr(self, "h", None):
            _destroy(self.h)
            self.h = None

    def set_particles(self, xyz, alpha: float) -> None:
        x = np.ascontiguousarray(xyz, np.float64).reshape(-1, 3)
        self.n = len(x)
        self.alpha = float(alpha)
        check(lib.PfemLoop_set_particles(self.h, len(x), _p(x), alpha), "PfemLoop_set_particles")

    def particles(self) -> np.ndarray:
        x = np.empty((self.n, 3), np.float64)
        check(lib.PfemLoop_get_particles(self.h, _p(x)), "PfemLoop_get_particles")
        return x

    def set_flow(self, flow: TaylorGreen) -> None:
        self.flow = flow
        check(lib.PfemLoop_set_flow(self.h, _p(flow.packed())), "PfemLoop_set_flow")

    def set_physics(self, physics: Physics | None) -> None:
        """Fractional-step dynamics instead of the Taylor-Green advection (None: off)."""
        self.physics = physics
        check(lib.PfemLoop_set_physics(self.h, _p(physics.packed()) if physics is not None else None),
              "PfemLoop_set_physics")

    def velocity(self) -> np.ndarray:
        u = np.empty((self.n, 3), np.float64)
        check(lib.PfemLoop_get_velocity(self.h, _p(u)), "PfemLoop_get_velocity")
        return u

    def set_velocity(self, u: np.ndarray) -> None:
        v = np.ascontiguousarray(u, np.float64).reshape(-1, 3)
        if len(v) != self.n:
            raise ValueError(f"set_velocity: {len(v)} values for {self.n} particles")
        check(lib.PfemLoop_set_velocity(self.h, _p(v)), "PfemLoop_set_velocity")

    def set_fsai(self, model: FsaiModel | None) -> None:
        self._model = model
        check(lib.PfemLoop_set_fsai(self.h, model.h if model is not None else None), "PfemLoop_set_fsai")

    def step(self, dt: float, rtol: float = 1e-8) -> dict:
        rep = np.zeros(12, np.float64)
        check(lib.PfemLoop_step(self.h, dt, rtol, _p(rep)), "PfemLoop_step")
        out = dict(zip(REPORT_KEYS, rep.tolist()))
        for k in ("iterations", "nodes", "tets"):
            out[k] = int(out[k])
        out["fallback"] = bool(out["fallback"])
        out["converged"] = bool(out["converged"])
        return out

    def pressure(self) -> np.ndarray:
        p = np.empty(self.n, np.float64)
        check(lib.PfemLoop_get_pressure(self.h, _p(p)), "PfemLoop_get_pressure")
        return p

    def set_pressure(self, p: np.ndarray) -> None:
        """Initial guess of the next solve (particle order); each step otherwise
        starts from the previous step's pressure."""
        q = np.ascontiguousarray(p, np.float64).reshape(-1)
        if len(q) != self.n:
            raise ValueError(f"set_pressure: {len(q)} values for {self.n} particles")
        check(lib.PfemLoop_set_pressure(self.h, _p(q)), "PfemLoop_set_pressure")

    def stats(self) -> dict:
        st = np.zeros(2, np.uint64)
        check(lib.PfemLoop_stats(self.h, _p(st)), "PfemLoop_stats")
        return {"steps": int(st[0]), "fallback_steps": int(st[1])}

    # ---- checkpoint / resume: particle positions, the field, the step count,
    # the last pressure (the next solve's initial guess; None before the first
    # step) and, with the fractional-step dynamics, the velocities and parameters
    def save(self, path: str, step: int) -> None:
        try:  # the pressure the next solve starts from: the last step's, or one set_pressure() gave
            p = self.pressure()
        except StreamError:
            p = np.zeros(0)
        ph = getattr(self, "physics", None)
        np.savez(path, xyz=self.particles(), alpha=self.alpha, flow=self.flow.packed(), step=step, pressure=p,
                 velocity=self.velocity() if ph is not None else np.zeros(0),
                 physics=ph.packed() if ph is not None else np.zeros(0))

    @staticmethod
    def load_dynamics(path: str):
        """(velocity or None, Physics or None) of a checkpoint saved with the
        fractional-step dynamics on (None, None otherwise)."""
        d = np.load(path)
        if "physics" not in d or not len(d["physics"]):
            return None, None
        q = d["physics"]
        return d["velocity"], Physics(q[0:3], q[3], q[4], q[5:8], q[8:11])

    @staticmethod
    def load(path: str):
        """(xyz, alpha, flow, step, pressure or None) of a checkpoint."""
        d = np.load(path)
        f = d["flow"]
        flow = TaylorGreen(f[:9].reshape(3, 3), f[9:12], f[12], f[13])
        p = d["pressure"] if "pressure" in d and len(d["pressure"]) else None
        return d["xyz"], float(d["alpha"]), flow, int(d["step"]), p
