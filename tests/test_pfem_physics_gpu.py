"""GPU: the fractional-step dynamics of the PFEM loop (PfemLoop_set_physics):
Chorin's projection on the P1 mesh of the particles with gravity, viscosity
and box walls.  The reference has no such step, so the checks are physical
and analytic: hydrostatic pressure in a tank at rest, exact transport of a
divergence-free linear velocity field, removal of the divergence of an
expanding one, and a dam break that stays bounded and spreads."""
import numpy as np
import pytest

from stream_b200 import workloads

pytestmark = pytest.mark.gpu


def _loop(pts, h, physics, alpha=1.2):
    from stream_b200.pfem import PfemLoop
    L = PfemLoop(pts.astype(np.float64), alpha * h)
    L.set_physics(physics)
    return L


def test_tank_at_rest_is_hydrostatic():
    """A column filling its tank's width: after one step from rest the
    pressure is rho g (y_top - y) and the fluid stays (nearly) at rest."""
    from stream_b200.pfem import Physics
    h = 0.02
    pts, _ = workloads.dambreak_column(h=h, seed=1, extent=(0.2, 0.4, 0.2))
    ph = Physics(g=(0, -9.81, 0), nu=0.0, rho=1000.0, lo=(0, 0, 0), hi=(0.2, 0.8, 0.2))
    L = _loop(pts, h, ph)
    dt = 1e-3
    rep = L.step(dt, rtol=1e-10)
    assert rep["converged"]
    p = L.pressure()
    y = pts[:, 1].astype(np.float64)
    ytop = y.max()
    want = 1000.0 * 9.81 * (ytop - y)
    inner = (y < ytop - 1.5 * h)
    rel = np.abs(p[inner] - want[inner]) / want[inner]
    assert np.median(rel) < 0.05, np.median(rel)
    assert np.corrcoef(p[inner], want[inner])[0, 1] > 0.99
    u = L.velocity()
    mid = (y > 3 * h) & (y < ytop - 3 * h)
    assert np.abs(u[mid]).max() < 0.25 * 9.81 * dt, np.abs(u[mid]).max()


def test_divergence_free_linear_field_is_transported_exactly():
    """u = (x - cx, -(y - cy), 0), no gravity, no viscosity, walls far away:
    the pressure load vanishes, so every particle moves by dt u."""
    from stream_b200.pfem import Physics
    h = 0.02
    pts, _ = workloads.dambreak_column(h=h, seed=2, extent=(0.2, 0.2, 0.2))
    x0 = pts.astype(np.float64)
    c = x0.mean(0)
    u0 = np.stack([x0[:, 0] - c[0], -(x0[:, 1] - c[1]), np.zeros(len(x0))], 1)
    L = _loop(pts, h, Physics(g=(0, 0, 0), nu=0.0, rho=1.0, lo=(-10, -10, -10), hi=(10, 10, 10)))
    L.set_velocity(u0)
    dt = 1e-3
    L.step(dt, rtol=1e-8)
    assert np.abs(L.particles() - (x0 + dt * u0)).max() < 1e-9
    assert np.abs(L.velocity() - u0).max() < 1e-6


def test_projection_removes_the_divergence_of_an_expanding_field():
    """u = x - c (divergence 3), no gravity or viscosity: the pressure is a
    suction (negative inside; zero only at the rare interior node next to a
    sliver the alpha shape drops, which it flags as free surface).  The
    projection is approximate (consistent divergence, lumped gradient, P1
    Laplacian): the fitted interior divergence falls from 3 to below 1, and a
    second step finds far less to remove."""
    from stream_b200.pfem import Physics
    h = 0.02
    pts, _ = workloads.dambreak_column(h=h, seed=3, extent=(0.24, 0.24, 0.24))
    x0 = pts.astype(np.float64)
    c = x0.mean(0)
    L = _loop(pts, h, Physics(g=(0, 0, 0), nu=0.0, rho=1.0, lo=(-10, -10, -10), hi=(10, 10, 10)))
    L.set_velocity(x0 - c)
    L.step(1e-3, rtol=1e-10)
    p1 = L.pressure()
    d = np.abs(x0 - c).max(1)
    inner = d < 0.12 - 2.5 * h
    assert np.all(p1[inner] <= 0) and np.mean(p1[inner] < 0) > 0.95
    u1 = L.velocity()[inner]
    X = np.concatenate([x0[inner] - c, np.ones((inner.sum(), 1))], 1)
    A = np.linalg.lstsq(X, u1, rcond=None)[0][:3].T  # u1 ~ A (x - c) + b
    assert abs(np.trace(A)) < 1.0, np.trace(A)
    L.step(1e-3, rtol=1e-10)
    p2 = L.pressure()
    assert np.abs(p2[inner]).max() < 0.35 * np.abs(p1[inner]).max(), (np.abs(p2[inner]).max(), np.abs(p1[inner]).max())


def test_dam_break_spreads_and_stays_in_the_tank():
    from stream_b200.pfem import Physics
    h = 0.02
    pts, _ = workloads.dambreak_column(h=h, seed=4, extent=(0.2, 0.4, 0.1))
    hi = np.array([0.8, 0.6, 0.1])
    L = _loop(pts, h, Physics(g=(0, -9.81, 0), nu=1e-6, rho=1000.0, lo=(0, 0, 0), hi=hi))
    y0 = pts[:, 1].mean()
    front = [float(pts[:, 0].max())]
    for _ in range(40):
        rep = L.step(2e-3, rtol=1e-8)
        assert rep["converged"]
        front.append(float(L.particles()[:, 0].max()))
    x = L.particles()
    u = L.velocity()
    assert np.isfinite(x).all() and np.isfinite(u).all()
    assert (x >= -1e-12).all() and (x <= hi + 1e-12).all()
    assert front[-1] > front[0] + 1.5 * h, front           # the front has moved out
    assert x[:, 1].mean() < y0 - 0.01                      # the column has come down
    assert np.abs(u).max() < 2.0 * np.sqrt(2 * 9.81 * 0.4)  # bounded by the fall speed


def test_physics_parameters_are_checked():
    from stream_b200 import StreamError
    from stream_b200.pfem import Physics
    pts, _ = workloads.dambreak_column(h=0.05, seed=5, extent=(0.2, 0.2, 0.2))
    from stream_b200.pfem import PfemLoop
    L = PfemLoop(pts.astype(np.float64), 0.06)
    with pytest.raises(StreamError):
        L.set_physics(Physics(rho=0.0))
    with pytest.raises(StreamError):
        L.set_physics(Physics(lo=(1, 0, 0), hi=(0, 1, 1)))
    with pytest.raises(ValueError):
        L.set_velocity(np.zeros((3, 3)))


def test_checkpoint_resume_keeps_the_dynamics(tmp_path):
    """save() stores velocities and parameters; a loop rebuilt from the
    checkpoint continues like the original (the pressure solves agree to
    their tolerance: FP64 atomic dot products may round in another order)."""
    from stream_b200.pfem import PfemLoop, Physics
    h = 0.02
    pts, _ = workloads.dambreak_column(h=h, seed=6, extent=(0.2, 0.3, 0.1))
    L = _loop(pts, h, Physics(g=(0, -9.81, 0), nu=1e-6, rho=1000.0, lo=(0, 0, 0), hi=(0.6, 0.5, 0.1)))
    for _ in range(3):
        L.step(2e-3, rtol=1e-10)
    L.save(str(tmp_path / "d.npz"), step=3)
    xyz, alpha, flow, step, p = PfemLoop.load(str(tmp_path / "d.npz"))
    u, ph = PfemLoop.load_dynamics(str(tmp_path / "d.npz"))
    assert step == 3 and ph is not None and np.array_equal(ph.packed(), L.physics.packed())
    R = PfemLoop(xyz, alpha, flow)
    R.set_physics(ph)
    R.set_velocity(u)
    R.set_pressure(p)
    for _ in range(2):
        L.step(2e-3, rtol=1e-10)
        R.step(2e-3, rtol=1e-10)
    assert np.abs(R.particles() - L.particles()).max() < 1e-9
    assert np.abs(R.velocity() - L.velocity()).max() < 1e-6 * max(1.0, np.abs(L.velocity()).max())
