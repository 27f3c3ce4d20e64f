"""Failure detection on host-crafted inputs (nothing here faults or hangs a
GPU: every case is rejected on the host or ends a bounded device loop with a
status the host reads).

* non-finite coordinates or alpha radii are refused by set_nodes before any
  meshing kernel runs (STREAM_ST_BAD_INPUT), in 3D (checked on the GPU copy
  of the input) and 2D (checked on the host);
* a Jacobi preconditioner over rows without a usable diagonal reports them
  (the reference would use an uninitialised inverse,
  src/numerics/preconditioner_jacobi.cpp:43-48), and the FP32 CG over such a
  matrix ends with a breakdown instead of running to its cap;
* singular systems end with converged = false inside the iteration cap;
* a deep LBVH (point pairs converging on one point, all of them inside the
  search radius) keeps the traversal inside its 64-entry stack and matches
  the oracle.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("where", ["coord_nan", "coord_inf", "alpha_nan", "alpha_inf"])
def test_set_nodes_rejects_non_finite_3d(sb, where):
    from stream_b200 import StreamError, STREAM_ST_BAD_INPUT, libmesh
    from stream_b200.mesh import AlphaShape3D
    rng = np.random.default_rng(0)
    pts = rng.random((500, 3)).astype(np.float32)
    al = np.full(500, 0.1, np.float32)
    bad = {"coord_nan": (pts, 17, 1, np.nan), "coord_inf": (pts, 3, 2, -np.inf),
           "alpha_nan": (al, 40, None, np.nan), "alpha_inf": (al, 0, None, np.inf)}[where]
    arr, i, j, v = bad
    if j is None:
        arr[i] = v
    else:
        arr[i, j] = v
    a = AlphaShape3D()
    with pytest.raises(StreamError, match="bad_input"):
        a.set_nodes(pts, al)
    assert libmesh.AlphaShape3D_get_status(a.mesh) & STREAM_ST_BAD_INPUT
    # the handle holds no nodes afterwards: a compute() is refused, not run on old data
    with pytest.raises(StreamError):
        a.compute()
    # and a valid point set afterwards meshes normally
    a.set_nodes(rng.random((500, 3)).astype(np.float32), np.full(500, 0.1, np.float32))
    a.compute()
    assert len(a.get_elem()) > 0


def test_set_nodes_rejects_non_finite_2d(sb):
    from stream_b200 import StreamError
    from stream_b200.mesh import AlphaShape2D
    rng = np.random.default_rng(1)
    pts = rng.random((400, 2)).astype(np.float32)
    al = np.full(400, 0.1, np.float32)
    pts[5, 0] = np.inf
    m = AlphaShape2D()
    with pytest.raises(StreamError):
        m.set_nodes(pts, al)


def _laplacian_1d(n, diag=2.0):
    rows, cols, vals = [], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, diag), (i + 1, -1.0)):
            if 0 <= j < n:
                rows.append(i)
                cols.append(j)
                vals.append(v)
    row = np.searchsorted(np.array(rows), np.arange(n + 1)).astype(np.uint32)
    return row, np.array(cols, np.uint32), np.array(vals, np.float64)


def test_jacobi_zero_and_missing_diagonal(sb):
    from stream_b200.numerics import DeviceCSR, HostCSR, LinSys, PrecJacobi, SolverCG
    n = 200
    row, col, val = _laplacian_1d(n)
    val = val.astype(np.float32)
    good = PrecJacobi(DeviceCSR(HostCSR(row, col, val)))
    assert good.bad_rows() == 0
    # one explicit zero on the diagonal, one row whose diagonal entry is absent
    v2 = val.copy()
    v2[np.nonzero((np.repeat(np.arange(n), np.diff(row)) == 50) & (col == 50))[0]] = 0.0
    keep = ~((np.repeat(np.arange(n), np.diff(row)) == 120) & (col == 120))
    r2 = np.concatenate([[0], np.cumsum(np.bincount(np.repeat(np.arange(n), np.diff(row))[keep], minlength=n))])
    dcsr = DeviceCSR(HostCSR(r2.astype(np.uint32), col[keep], v2[keep]))
    prec = PrecJacobi(dcsr)
    assert prec.bad_rows() == 2
    sys_ = LinSys(dcsr, np.ones(n, np.float32))
    solver = SolverCG()
    x = np.zeros(n, np.float32)
    it = solver.solve_jacobi(sys_, prec, x)
    assert solver.termination() == "breakdown"
    assert it < 10000


def test_singular_systems_stop_unconverged(sb):
    """Pure-Neumann 1D Laplacian (singular) with a right-hand side outside its
    range: FP64 Jacobi-PCG and mixed refinement stop at the cap, unconverged."""
    from stream_b200.numerics import PoissonSystem
    n = 300
    row, col, val = _laplacian_1d(n)
    # Neumann ends: diagonal 1 in the first and last rows, so constants are in the null space
    first = np.nonzero(col[: row[1]] == 0)[0][0]
    last = row[n - 1] + np.nonzero(col[row[n - 1]:row[n]] == n - 1)[0][0]
    val[first] = 1.0
    val[last] = 1.0
    b = np.ones(n)  # not orthogonal to the null space: no solution
    ps = PoissonSystem()
    ps.set_csr(row, col, val, b)
    for method in (PoissonSystem.FP64_JACOBI, PoissonSystem.MIXED_IR):
        x, rep = ps.solve(method=method, rtol=1e-8, maxit=400)
        assert not rep["converged"], (method, rep)
        assert rep["iterations"] <= 400 + 64, (method, rep)  # the cap, checked per batch of iterations


def test_deep_tree_stays_in_stack(sb, restate):
    from stream_b200 import workloads
    from stream_b200.mesh import AlphaShape3D
    pts, al = workloads.deep_spine()
    want = restate.ashape3d(pts, al)
    assert not (want.status & 1)
    a = AlphaShape3D()
    a.set_nodes(pts, al)
    a.compute()
    assert not (a.status & 1), f"status 0x{a.status:x}"
    assert np.array_equal(a.get_permutation(), want.perm)
    nineig, _, _ = a.get_stars()
    assert np.array_equal(nineig, want.nineig)
    assert np.array_equal(a.get_elem(), want.elems)


def test_lbvh_flags_non_finite_sphere(sb):
    """Host arrays through Sphere3DLBVH.set_objects are copied as given; a
    non-finite sphere is flagged by the global-box pass (ST_BAD_INPUT) and the
    build returns that status instead of an error-free tree."""
    from stream_b200 import STREAM_ST_BAD_INPUT
    from stream_b200.geometry import Sphere3DLBVH
    rng = np.random.default_rng(3)
    xyzr = np.concatenate([rng.random((1000, 3)), np.full((1000, 1), 0.01)], 1).astype(np.float32)
    xyzr[10, 3] = np.nan
    b = Sphere3DLBVH()
    b.set_objects(xyzr)
    st = b.build()
    assert st & STREAM_ST_BAD_INPUT
