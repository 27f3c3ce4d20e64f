"""Numerics on the GPU: the reference's FP32 CG / Jacobi-PCG API
(src/numerics/conjugate_gradient.cpp) against its known answers and the
reference build, and the FP64 / mixed-precision Poisson solves against SciPy
FP64 (tolerances are written per test)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from stream_b200 import workloads

pytestmark = pytest.mark.gpu


def _ref_solve(row, col, val, b, jacobi=True):
    import stream_b200.numerics as stn
    h = stn.HostCSR(row, col, val)
    d = stn.DeviceCSR(h)
    s = stn.LinSys(d, b)
    cg = stn.SolverCG()
    x = np.zeros(len(b), np.float32)
    if jacobi:
        it = cg.solve_jacobi(s, stn.PrecJacobi(d), x)
    else:
        it = cg.solve(s, x)
    return x, it


def test_cg_jacobi_diagonal_kat(sb, restate):
    """tests/numerics/cg_jacobi.cpp:36-83: diag(1..100) x = 1  ->  x_i = 1/i."""
    n = 100
    row = np.arange(n + 1, dtype=np.uint32)
    col = np.arange(n, dtype=np.uint32)
    val = np.arange(1, n + 1, dtype=np.float32)
    b = np.ones(n, np.float32)
    x, it = _ref_solve(row, col, val, b)
    assert np.max(np.abs(x - 1.0 / np.arange(1, n + 1))) <= 1e-7
    _, it_o = restate.cg_f32(row, col, val, b, np.zeros(n, np.float32))
    assert it == it_o == 0


def _python_cg_api_matrix(n=50_000, density=0.001, seed=42):
    """The random diagonally dominant SPD system of tests/numerics/python_cg_api.py:24-47."""
    nnz_half = int(n * (n * density)) // 2
    rs = np.random.RandomState(seed)
    r = rs.randint(0, n, size=(nnz_half,))
    c = rs.randint(0, n, size=(nnz_half,))
    v = rs.uniform(0, 1, size=(nnz_half,))
    A = sp.coo_array((v, (r, c)), shape=(n, n), dtype=np.float32)
    A = 0.5 * (A + A.T)
    A = sp.csr_array(A)
    A = A + sp.diags(A @ np.ones(n))
    A = sp.csr_array(A, dtype=np.float32)
    A.sort_indices()
    b = rs.uniform(0, 1, size=(n,)).astype(np.float32)
    return A, b


@pytest.mark.parametrize("jacobi", [True, False])
def test_cg_random_spd_vs_scipy(sb, restate, jacobi):
    A, b = _python_cg_api_matrix()
    x, it = _ref_solve(A.indptr.astype(np.uint32), A.indices.astype(np.uint32), A.data, b, jacobi)
    # FP64 reference solution by SciPy CG (the comparison tests/numerics/python_cg_api.py
    # makes); the matrix is strongly diagonally dominant, so CG converges fast.
    A64 = A.astype(np.float64)
    x64, info = spla.cg(A64, b.astype(np.float64), rtol=1e-13, maxiter=10000,
                        M=sp.diags(1.0 / A64.diagonal()))
    assert info == 0
    # FP32 recurrence with the reference's absolute stop sqrt(r.z) <= 1e-6.
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-5
    _, it_o = restate.cg_f32(A.indptr, A.indices, A.data, b, np.zeros(len(b), np.float32), jacobi=jacobi)
    assert abs(it - it_o) <= 2


def test_cg_vs_reference_build(sb, reference):
    A, b = _python_cg_api_matrix(n=20_000, seed=7)
    x, it = _ref_solve(A.indptr.astype(np.uint32), A.indices.astype(np.uint32), A.data, b)
    xr, itr = reference.cg_f32(A.indptr, A.indices, A.data, b, np.zeros(len(b), np.float32))
    assert abs(it - itr) <= 2
    assert np.linalg.norm(x - xr) / np.linalg.norm(xr) < 1e-5


def _mesh(pts, al):
    from stream_b200.mesh import AlphaShape3D
    m = AlphaShape3D()
    m.set_nodes(pts, al)
    m.compute()
    return m


def _p1_oracle(nodes, elems, is_bnd, modes=None):
    """NumPy FP64 P1 Laplacian with Dirichlet elimination (the new assembly
    has no reference counterpart; this is its oracle)."""
    n = len(nodes)
    X = nodes.astype(np.float64)[elems]                # (E, 4, 3)
    e1, e2, e3 = X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]
    det = np.einsum("ij,ij->i", e1, np.cross(e2, e3))
    ok = det != 0
    g = np.zeros((len(elems), 4, 3))
    g[:, 1] = np.cross(e2, e3) / det[:, None]
    g[:, 2] = np.cross(e3, e1) / det[:, None]
    g[:, 3] = np.cross(e1, e2) / det[:, None]
    g[:, 0] = -(g[:, 1] + g[:, 2] + g[:, 3])
    vol = np.abs(det) / 6.0
    K = vol[:, None, None] * np.einsum("eik,ejk->eij", g, g)
    K[~ok] = 0
    rows = np.repeat(elems, 4, axis=1).ravel()
    cols = np.tile(elems, (1, 4)).ravel()
    A = sp.csr_matrix((K.ravel(), (rows, cols)), shape=(n, n))
    if modes is None:
        f = np.ones(len(elems))
    else:
        c = X.mean(axis=1)
        f = np.zeros(len(elems))
        for kx, ky, kz, ak, ph in modes:
            f += ak * np.cos(kx * c[:, 0] + ky * c[:, 1] + kz * c[:, 2] + ph)
    bvec = np.zeros(n)
    np.add.at(bvec, elems.ravel(), np.repeat(0.25 * vol * f * ok, 4))
    deg = np.bincount(elems.ravel(), minlength=n)
    dirich = (is_bnd != 0) | (deg == 0)
    keep = ~dirich
    D = sp.diags(keep.astype(float))
    A = (D @ A @ D).tocsr() + sp.diags(dirich.astype(float))
    bvec[dirich] = 0.0
    return A, bvec


def test_assembly_vs_numpy(sb):
    pts, al = workloads.dambreak_column(h=0.02, seed=3)
    m = _mesh(pts, al)
    from stream_b200.numerics import PoissonSystem
    ps = PoissonSystem()
    ps.assemble(m)
    row, col, val, b = ps.get_csr()
    nodes = m.get_ordered_nodes()
    A0, b0 = _p1_oracle(nodes, m.get_elem().astype(np.int64), m.get_boundary_nodes())
    A = sp.csr_matrix((val, col, row), shape=A0.shape)
    diff = abs(A - A0)
    assert diff.max() <= 1e-12 * abs(A0).max()
    assert np.max(np.abs(b - b0)) <= 1e-12 * np.max(np.abs(b0))
    # Columns are sorted and the matrix is symmetric.
    for i in range(0, len(row) - 1, 97):
        c = col[row[i]:row[i + 1]]
        assert np.all(np.diff(c.astype(np.int64)) > 0)
    assert abs(A - A.T).max() <= 1e-14 * abs(A).max()


def _modes(seed=0, h=0.02):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(8):
        k = rng.integers(-3, 4, size=3) * np.pi
        a = rng.standard_normal(3)
        out.append([k[0], k[1], k[2], float(a @ k), rng.uniform(0, 2 * np.pi)])
    return np.array(out, np.float32)


@pytest.mark.parametrize("method", [0, 1])
@pytest.mark.parametrize("rhs", ["one", "div"])
def test_poisson_solve_vs_scipy(sb, method, rhs):
    pts, al = workloads.dambreak_column(h=0.02, seed=4)
    m = _mesh(pts, al)
    from stream_b200.numerics import PoissonSystem
    ps = PoissonSystem()
    modes = _modes() if rhs == "div" else None
    ps.assemble(m, rhs="one" if rhs == "one" else "div", modes=modes)
    row, col, val, b = ps.get_csr()
    A = sp.csr_matrix((val, col, row), shape=(len(b), len(b)))
    x64 = spla.spsolve(A.tocsc(), b)
    x, rep = ps.solve(method=method, rtol=1e-8)
    assert rep["converged"]
    # True FP64 relative residual reported by the solver and recomputed here.
    rr = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert rep["relres"] <= 1e-8 and rr <= 1e-8
    assert abs(rr - rep["relres"]) <= 1e-3 * max(rr, 1e-300) + 1e-15
    # ||x - x64|| / ||x64|| <= cond(A) * 1e-8; cond ~ (1/h)^2 = 2500 here.
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) <= 5e-5


def _far_and_long_rows(n=70000, seed=0):
    """SPD matrix with columns far from their row (> 32767 apart) and a band
    of long rows (rows 5000..5199 couple to 150 random columns each), unlike
    the short, near-diagonal rows of a Morton-ordered mesh."""
    rng = np.random.default_rng(seed)
    i = np.arange(n)
    rows = [i[:-1], i[:-3]]
    cols = [i[1:], i[3:]]
    far = rng.choice(n, 4000, replace=False)
    rows.append(far)
    cols.append((far + rng.integers(33000, 60000, far.size)) % n)
    long_r = np.repeat(np.arange(5000, 5200), 150)
    rows.append(long_r)
    cols.append(rng.integers(0, n, long_r.size))
    r = np.concatenate(rows)
    c = np.concatenate(cols)
    keep = r != c
    r, c = r[keep], c[keep]
    w = rng.uniform(0.1, 1.0, r.size)
    L = sp.coo_matrix((-w, (r, c)), shape=(n, n)).tocsr()
    L = L + L.T
    L.sum_duplicates()
    A = (L - sp.diags(np.asarray(L.sum(axis=1)).ravel() - 0.05)).tocsr()  # diagonally dominant, SPD
    A.sort_indices()
    return A


@pytest.mark.parametrize("method", [0, 1, 2, 3])
def test_solves_far_columns_and_long_rows(sb, method):
    """All four solvers on a matrix unlike a mesh's (set from host CSR, no
    coordinates for the learned preconditioner's geometric features; the
    Kolotilina-Yeremin pass leaves the 150-entry rows diagonal)."""
    from stream_b200.numerics import FsaiModel, PoissonSystem
    A = _far_and_long_rows()
    n = A.shape[0]
    d = np.abs(A.indices.astype(np.int64) - np.repeat(np.arange(n), np.diff(A.indptr)))
    assert (d > 32767).sum() > 1000 and np.diff(A.indptr).max() >= 150
    b = np.random.default_rng(1).normal(size=n)
    ps = PoissonSystem()
    ps.set_csr(A.indptr, A.indices, A.data, b)
    if method == 2:
        ps.set_fsai(FsaiModel.trained())
    x, rep = ps.solve(method=method, rtol=1e-8)
    assert rep["converged"] and not rep["fallback"], rep
    rr = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert rr <= 1e-8 and rep["relres"] <= 1e-8
