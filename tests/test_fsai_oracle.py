"""The learned-FSAI oracle (oracle/fsai_oracle.py) on the CPU: its analytic
gradients (both losses) against central finite differences, the Kaporin loss
against its closed form and its ordering of Jacobi vs the Kolotilina-Yeremin
factor, the Jacobi identity of a zero output layer, SPD-ness of M = G^T G,
and its bfloat16 rounding against torch's.  The reference has no learned
preconditioner, so these checks are what pins the oracle."""
import numpy as np
import pytest

from oracle import fsai_oracle as fo
from tests.fsai_cases import grid_system


@pytest.fixture(scope="module")
def system():
    row, col, val, xyz = grid_system(4, seed=1)
    return fo.System(row, col, val, xyz)


@pytest.mark.parametrize("kind", ["residual", "kaporin"])
def test_gradient_matches_finite_differences(system, kind):
    vec = fo.init_params(3, last_scale=0.5).astype(np.float64)
    Z = fo.probes(system.n, 16, 11)
    L, g, _ = system.loss_and_grad(vec, Z, rounding=False, kind=kind)
    assert np.isfinite(L) and (L > 0 or kind == "kaporin")
    rng = np.random.default_rng(5)
    eps = 1e-6
    for _ in range(3):  # random directions
        dv = rng.standard_normal(fo.PARAM_COUNT)
        fd = (system.loss(vec + eps * dv, Z, False, kind) - system.loss(vec - eps * dv, Z, False, kind)) / (2 * eps)
        assert abs(fd - g @ dv) <= 1e-6 * max(1.0, abs(fd))
    for i in rng.integers(0, fo.PARAM_COUNT, 12):  # single coordinates
        e = np.zeros(fo.PARAM_COUNT)
        e[i] = eps
        fd = (system.loss(vec + e, Z, False, kind) - system.loss(vec - e, Z, False, kind)) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd)


def _ky_fsai(system):
    """Kolotilina-Yeremin factor on the lower pattern of A: row i solves
    A[P, P] g = e_i over its lower pattern P, scaled to g_i = 1/sqrt(g_i)."""
    A = system.A.toarray()
    G = np.zeros_like(A)
    for i in range(system.n):
        P = system.c[system.r == i]
        g = np.linalg.solve(A[np.ix_(P, P)], (P == i).astype(float))
        G[i, P] = g / np.sqrt(g[P == i][0])
    return G


def test_kaporin_loss_closed_form_and_ky_minimum(system):
    import scipy.sparse as sp
    n = system.n
    Z = np.sqrt(n) * np.eye(n)  # n probes sqrt(n) e_p: the estimate is the exact trace
    jac = sp.diags(1.0 / np.sqrt(system.d))
    ky = sp.csr_matrix(_ky_fsai(system))
    for Gm in (jac, ky):
        L, _ = fo.kaporin_loss_and_dG(system.A, Gm.tocsr(), system.r, system.c, Z)
        M = (Gm @ system.A @ Gm.T).toarray()
        want = np.log(np.trace(M) / n) - 2.0 / n * np.log(Gm.diagonal()).sum()
        assert abs(L - want) <= 1e-12 * max(1.0, abs(want))
    Lj = fo.kaporin_loss_and_dG(system.A, jac.tocsr(), system.r, system.c, Z)[0]
    Lk = fo.kaporin_loss_and_dG(system.A, ky, system.r, system.c, Z)[0]
    assert Lk < Lj  # the KY factor minimises Kaporin's number over the pattern
    # ... and is a stationary point: the gradient on the free rows' entries vanishes
    _, dG = fo.kaporin_loss_and_dG(system.A, ky, system.r, system.c, Z)
    assert np.abs(dG[system.free[system.r]]).max() <= 1e-9


def test_zero_output_layer_is_jacobi(system):
    G, _ = system.g(fo.init_params(2, last_scale=0.0))
    want = np.where(system.r == system.c, 1.0 / np.sqrt(system.d[system.c]), 0.0)
    assert np.array_equal(G, want)


def test_m_is_spd_for_any_output(system):
    vec = fo.init_params(4, last_scale=5.0)  # large, arbitrary outputs
    G, _ = system.g(vec)
    Gm = fo.g_matrix(system.n, system.r, system.c, G).toarray()
    assert np.all(np.diag(Gm) > 0) and np.allclose(Gm, np.tril(Gm))
    assert np.linalg.eigvalsh(Gm.T @ Gm).min() > 0


def test_features_of_dirichlet_and_eliminated_entries(system):
    F, r, c = system.F, system.r, system.c
    fixed = ~system.free[r]
    assert np.all(F[fixed & (r == c), 7] == 1.0)  # identity rows: boundary fraction 1
    assert np.all((F[:, 7] >= 0) & (F[:, 7] <= 1))
    assert np.all(F[r == c, 9] == 1) and np.all(F[r != c, 9] == 0)
    assert abs(np.mean(F[(r != c) & (system.val[system.k] != 0), 6]) - 1.0) < 1e-12  # distances over h


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(10000) * 10.0 ** rng.integers(-6, 6, 10000),
                        [0.0, -0.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 65504.0]]).astype(np.float32)
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(fo.bf16(x).astype(np.float32), want)


def test_probes_are_rademacher():
    Z = fo.probes(1000, 16, 123)
    assert set(np.unique(Z)) == {-1.0, 1.0}
    assert abs(Z.mean()) < 0.05
    assert np.array_equal(Z, fo.probes(1000, 16, 123)) and not np.array_equal(Z, fo.probes(1000, 16, 124))


def test_ky_fsai_oracle_normalises_and_matches_dense_inverse():
    """The Kolotilina-Yeremin G: diag(G A G^T) = 1, and on a pattern that is
    the whole lower triangle it is the Cholesky factor of A^-1 (G^T G = A^-1)."""
    import scipy.sparse as sp
    from tests.fsai_cases import grid_system
    row, col, val, _ = grid_system(5, 1)
    n = len(row) - 1
    r, c, _ = fo.lower_edges(row, col)
    G = sp.csr_matrix((fo.ky_fsai(row, col, val), (r, c)), shape=(n, n))
    A = sp.csr_matrix((val, col, row), shape=(n, n))
    assert np.max(np.abs((G @ A).multiply(G).sum(1).A1 - 1.0)) <= 1e-12
    rng = np.random.default_rng(0)
    B = rng.standard_normal((12, 12))
    D = B @ B.T + 12 * np.eye(12)
    Ds = sp.csr_matrix(D)
    Ds.sort_indices()
    rr, cc, _ = fo.lower_edges(Ds.indptr, Ds.indices)
    Gd = sp.csr_matrix((fo.ky_fsai(Ds.indptr, Ds.indices, Ds.data), (rr, cc)), shape=(12, 12)).toarray()
    assert np.allclose(Gd.T @ Gd, np.linalg.inv(D), atol=1e-12)
