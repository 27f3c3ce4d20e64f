"""PFEM step loop on the GPU: the advection kernel against a NumPy FP64
restatement of the same Euler steps, every step's solve against the FP64
tolerance, the loop's pressure against an independent remesh + assembly +
SciPy solve of the same particles, and checkpoint/resume."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from stream_b200 import workloads

pytestmark = pytest.mark.gpu


def _modes(seed=0):
    rng = np.random.default_rng(seed)
    k = rng.normal(size=(8, 3)) * 6.0
    amp = rng.normal(size=(8, 3))
    return np.concatenate([k, np.sum(amp * k, 1, keepdims=True), rng.uniform(0, 6.28, (8, 1))], 1).astype(np.float32)


def test_advection_matches_numpy(sb):
    from stream_b200.pfem import TaylorGreen, advect_taylor_green
    rng = np.random.default_rng(0)
    x0 = rng.uniform(0, 1, (20000, 3))
    flow = TaylorGreen.random(rng)
    got = advect_taylor_green(x0, flow, 0.005, 7)
    want = x0.copy()
    for _ in range(7):
        want = want + 0.005 * flow.velocity(want)
    assert np.abs(got - want).max() <= 1e-13
    # divergence-free field: the volume of a small cube is kept to O(dt^2)
    c = np.array([[0.3, 0.4, 0.5]]) + 1e-4 * np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]])
    c1 = advect_taylor_green(c, flow, 0.005, 1)
    v0 = np.linalg.det(c[1:] - c[0])
    v1 = np.linalg.det(c1[1:] - c1[0])
    assert abs(v1 / v0 - 1) < 1e-3


def _loop(model=None, h=0.03, seed=1):
    from stream_b200.pfem import PfemLoop, TaylorGreen
    pts, al = workloads.dambreak_column(h=h, seed=seed)
    return PfemLoop(pts.astype(np.float64), float(al[0]), TaylorGreen(amp=0.5), _modes(seed), model)


@pytest.mark.parametrize("with_model", [False, True])
def test_steps_converge(sb, with_model):
    from stream_b200.numerics import FsaiModel
    model = FsaiModel.trained() if with_model else None
    L = _loop(model)
    for _ in range(3):
        r = L.step(0.002)
        assert r["converged"] and r["relres"] <= 1e-8 and not r["fallback"], r
        assert r["nodes"] == L.n and r["tets"] > 0
        assert r["step_ms"] >= r["solve_ms"] > 0
    p = L.pressure()
    assert np.all(np.isfinite(p)) and np.abs(p).max() > 0
    assert L.stats() == {"steps": 3, "fallback_steps": 0}


def test_pressure_matches_independent_solve(sb):
    from stream_b200.mesh import AlphaShape3D
    from stream_b200.numerics import PoissonSystem
    L = _loop()
    L.step(0.002)
    x = L.particles()
    p = L.pressure()
    a = AlphaShape3D()
    a.set_nodes(x.astype(np.float32), np.full(len(x), L.alpha, np.float32))
    a.compute()
    ps = PoissonSystem()
    ps.assemble(a, rhs="div", modes=_modes(1))
    row, col, val, b = ps.get_csr()
    A = sp.csr_matrix((val, col, row), shape=(len(b), len(b)))
    pm = spla.spsolve(A.tocsc(), b)
    perm = a.get_permutation()
    want = np.empty_like(pm)
    want[perm] = pm
    assert np.linalg.norm(p - want) / np.linalg.norm(want) <= 1e-6


def test_checkpoint_resume(sb, tmp_path):
    from stream_b200.pfem import PfemLoop
    L = _loop()
    for _ in range(2):
        L.step(0.002)
    L.save(str(tmp_path / "ck.npz"), step=2)
    for _ in range(2):
        L.step(0.002)
    xyz, alpha, flow, step, p = PfemLoop.load(str(tmp_path / "ck.npz"))
    assert step == 2 and p is not None and len(p) == len(xyz)
    R = PfemLoop(xyz, alpha, flow, _modes(1))
    R.set_pressure(p)  # the continued loop starts its next solve from this pressure too
    for _ in range(2):
        R.step(0.002)
    assert np.array_equal(R.particles(), L.particles())  # advection is deterministic
    # same system; both solves stop at relative residual 1e-8 (dot products
    # accumulate with FP64 atomics, so their rounding order may differ)
    assert np.linalg.norm(R.pressure() - L.pressure()) <= 1e-6 * np.linalg.norm(L.pressure())


def test_checkpoint_resave_before_first_step_keeps_pressure(sb, tmp_path):
    """load() + set_pressure() + save() before any step keeps the pressure, so
    a second resume still warm-starts from it."""
    from stream_b200.pfem import PfemLoop
    L = _loop()
    L.step(0.002)
    L.save(str(tmp_path / "a.npz"), step=1)
    xyz, alpha, flow, step, p = PfemLoop.load(str(tmp_path / "a.npz"))
    R = PfemLoop(xyz, alpha, flow, _modes(1))
    R.set_pressure(p)
    R.save(str(tmp_path / "b.npz"), step=step)
    _, _, _, step2, p2 = PfemLoop.load(str(tmp_path / "b.npz"))
    assert step2 == 1 and p2 is not None and np.array_equal(p2, p)
