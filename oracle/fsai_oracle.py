"""NumPy oracle of the learned FSAI preconditioner (test infrastructure only).

The reference has no learned preconditioner, so there is nothing of it to pin
against: this module restates in float64 the arithmetic the CUDA path
(stream_b200/csrc/fsai.cu) implements, so that the GPU's features, G values,
loss and parameter gradients can be checked, and it is itself checked by
finite differences (tests/test_fsai_oracle.py).  Nothing in the product
imports it.

Definitions (A: symmetric CSR with sorted columns and a positive diagonal):

* lower edges: the entries (i, j), j <= i, of A in CSR order;
* per node: d_i = a_ii; bnd_i = (explicit zero off-diagonals of row i) /
  (off-diagonals of row i), and 1 for a row without off-diagonals or with
  only zero ones (a Dirichlet identity row or an isolated node);
  free_i = (bnd_i < 1); lmean = mean of log d_i over free rows (0 if none);
* h = mean |x_j - x_i| over strictly lower edges with a_ij != 0 (1 if none
  or without coordinates);
* features (16 wide, the last 6 zero): a_ij / sqrt(d_i d_j), log d_i - lmean,
  log d_j - lmean, (x_j - x_i) / h (3), |x_j - x_i| / h, bnd_i, bnd_j, [i == j];
* MLP 16 -> 64 -> 64 -> 64 -> 1, GELU in its tanh form
  0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))).  Inputs, the three weight
  matrices and the activations entering layers 2 and 3 are rounded to
  bfloat16 (the tensor-core operands); w4 is rounded to bfloat16 too; biases
  and accumulations are float32 on the GPU (float64 here);
* G (lower triangular): free row i: G_ii = exp(clip(o_ii, -4, 4)) / sqrt(d_i),
  G_ij = o_ij / sqrt(d_j) if a_ij != 0 else 0; non-free row: G_ii = 1/sqrt(d_i),
  G_ij = 0.  M = G^T G is SPD for every network output;
* losses over P probe vectors z_p (columns of Z):
  residual  L = sum_p ||G A G^T z_p - z_p||^2 / (P n);
  kaporin   L = log(t / n) - (2/n) sum_i log G_ii, t = sum_p z_p^T G A G^T z_p / P
  (t estimates tr(G A G^T), so L + log(det A)/n estimates the log of
  Kaporin's condition number of G A G^T, the functional that the
  Kolotilina-Yeremin FSAI minimises over the pattern);
* parameter gradients by the chain rule (the bfloat16 roundings count as
  identity in the derivative).

Parameters are one float32 vector of PARAM_COUNT values, in the order of
LAYOUT (matrices row-major, input index first).
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

NF = 16
HID = 64
LAYOUT = [("W1", (NF, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)),
          ("W3", (HID, HID)), ("b3", (HID,)), ("w4", (HID,)), ("b4", (1,))]
PARAM_COUNT = sum(int(np.prod(s)) for _, s in LAYOUT)
GELU_C0 = math.sqrt(2.0 / math.pi)
GELU_C1 = 0.044715
DIAG_CLIP = 4.0


def unpack(vec):
    vec = np.asarray(vec, dtype=np.float64)
    assert vec.shape == (PARAM_COUNT,)
    out, o = {}, 0
    for name, shape in LAYOUT:
        m = int(np.prod(shape))
        out[name] = vec[o:o + m].reshape(shape)
        o += m
    return out


def pack(params):
    return np.concatenate([np.asarray(params[name], np.float64).reshape(-1) for name, _ in LAYOUT])


def bf16(x):
    """Round to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64).reshape(a.shape)


def _identity(x):
    return np.asarray(x, dtype=np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + np.tanh(GELU_C0 * (z + GELU_C1 * z ** 3)))


def dgelu(z):
    t = np.tanh(GELU_C0 * (z + GELU_C1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C0 * (1.0 + 3.0 * GELU_C1 * z * z)


def lower_edges(row, col):
    """(rows, cols, positions) of the entries j <= i, in CSR order."""
    row = np.asarray(row, np.int64)
    col = np.asarray(col, np.int64)
    r = np.repeat(np.arange(len(row) - 1), np.diff(row))
    keep = col <= r
    return r[keep], col[keep], np.nonzero(keep)[0]


def node_info(row, col, val):
    n = len(row) - 1
    r = np.repeat(np.arange(n), np.diff(row))
    off = col != r
    d = np.zeros(n)
    diag = ~off
    d[r[diag]] = val[diag]
    n_off = np.bincount(r[off], minlength=n)
    n_zero = np.bincount(r[off & (val == 0)], minlength=n)
    bnd = np.ones(n)
    has = (n_off > 0) & (n_zero < n_off)
    bnd[has] = n_zero[has] / n_off[has]
    free = bnd < 1.0
    lmean = float(np.mean(np.log(d[free]))) if free.any() else 0.0
    return d, bnd, free, lmean


def features(row, col, val, xyz=None, ky=None):
    """(rows, cols, positions, F[E,16], d, bnd, free, h) of the lower edges;
    ky (the Kolotilina-Yeremin G on the lower edges) adds feature 10,
    K_ij sqrt(d_j)."""
    row = np.asarray(row, np.int64)
    col = np.asarray(col, np.int64)
    val = np.asarray(val, np.float64)
    d, bnd, free, lmean = node_info(row, col, val)
    r, c, k = lower_edges(row, col)
    a = val[k]
    F = np.zeros((len(r), NF))
    F[:, 0] = a / np.sqrt(d[r] * d[c])
    F[:, 1] = np.log(d[r]) - lmean
    F[:, 2] = np.log(d[c]) - lmean
    h = 1.0
    if xyz is not None:
        xyz = np.asarray(xyz, np.float64)
        dx = xyz[c] - xyz[r]
        dist = np.linalg.norm(dx, axis=1)
        sel = (r != c) & (a != 0)
        if sel.any():
            h = float(dist[sel].mean())
        F[:, 3:6] = dx / h
        F[:, 6] = dist / h
    F[:, 7] = bnd[r]
    F[:, 8] = bnd[c]
    F[:, 9] = (r == c)
    if ky is not None:
        F[:, 10] = np.asarray(ky, np.float64) * np.sqrt(d[c])
    return r, c, k, F, d, bnd, free, h


class MLP:
    def __init__(self, vec, rounding=True):
        self.p = unpack(vec)
        self.rd = bf16 if rounding else _identity

    def forward(self, F):
        p, rd = self.p, self.rd
        x = rd(F)
        z1 = x @ rd(p["W1"]) + p["b1"]
        z2 = rd(gelu(z1)) @ rd(p["W2"]) + p["b2"]
        z3 = rd(gelu(z2)) @ rd(p["W3"]) + p["b3"]
        h3 = gelu(z3)
        out = h3 @ rd(p["w4"]) + p["b4"][0]
        return out, (x, z1, z2, z3)

    def backward(self, cache, dout):
        p, rd = self.p, self.rd
        x, z1, z2, z3 = cache
        g = {}
        h3 = gelu(z3)
        g["w4"] = h3.T @ dout
        g["b4"] = np.array([dout.sum()])
        dz3 = np.outer(dout, rd(p["w4"])) * dgelu(z3)
        g["W3"] = rd(gelu(z2)).T @ dz3
        g["b3"] = dz3.sum(0)
        dz2 = (dz3 @ rd(p["W3"]).T) * dgelu(z2)
        g["W2"] = rd(gelu(z1)).T @ dz2
        g["b2"] = dz2.sum(0)
        dz1 = (dz2 @ rd(p["W2"]).T) * dgelu(z1)
        g["W1"] = x.T @ dz1
        g["b1"] = dz1.sum(0)
        return pack(g)


def g_values(out, r, c, a, d, free, ky=None):
    """G on the lower edges and dG/d(out) (0 where G does not depend on out).
    Without ky: G_ii = exp(out) / sqrt(d_i), G_ij = out / sqrt(d_j); with the
    Kolotilina-Yeremin G K: G_ii = exp(out) K_ii, G_ij = K_ij + out / sqrt(d_j)."""
    diag = r == c
    isd_c = 1.0 / np.sqrt(d[c])
    clipped = np.clip(out, -DIAG_CLIP, DIAG_CLIP)
    if ky is None:
        G = np.where(diag, np.exp(clipped) * isd_c, out * isd_c)
    else:
        K = np.asarray(ky, np.float64)
        G = np.where(diag, np.exp(clipped) * K, K + out * isd_c)
    dGdo = np.where(diag, np.where(np.abs(out) < DIAG_CLIP, G, 0.0), isd_c)
    off_zero = (~diag) & (a == 0)
    G = np.where(off_zero, 0.0, G)
    dGdo = np.where(off_zero, 0.0, dGdo)
    fixed = ~free[r]
    G = np.where(fixed, np.where(diag, isd_c, 0.0), G)
    dGdo = np.where(fixed, 0.0, dGdo)
    return G, dGdo


def g_matrix(n, r, c, G):
    return sp.csr_matrix((G, (r, c)), shape=(n, n))


def loss_and_dG(A, Gm, r, c, Z):
    """L = sum_p ||G A G^T z_p - z_p||^2 / (P n) and dL/dG on the lower edges."""
    n, P = Z.shape
    W = A @ (Gm.T @ Z)
    E = Gm @ W - Z
    L = float((E * E).sum() / (P * n))
    T = A @ (Gm.T @ E)
    dG = 2.0 / (P * n) * ((E[r] * W[c]).sum(1) + (Z[r] * T[c]).sum(1))
    return L, dG


def kaporin_loss_and_dG(A, Gm, r, c, Z):
    """L = log(t / n) - (2/n) sum_i log G_ii with t = sum_p z_p^T G A G^T z_p / P,
    and dL/dG on the lower edges: 2/(P t) sum_p Z_ip (A G^T Z)_jp, minus
    2/(n G_ii) on the diagonal."""
    n, P = Z.shape
    Y = Gm.T @ Z
    W = A @ Y
    ts = float((Y * W).sum())  # P t
    diag = Gm.diagonal()
    L = math.log(ts / (P * n)) - 2.0 / n * float(np.log(diag).sum())
    dG = 2.0 / ts * (Z[r] * W[c]).sum(1) - np.where(r == c, 2.0 / (n * diag[r]), 0.0)
    return L, dG


LOSSES = {"residual": loss_and_dG, "kaporin": kaporin_loss_and_dG}


def ky_fsai(row, col, val, max_len=24):
    """The Kolotilina-Yeremin FSAI on A's lower pattern, in float64: row i of G
    solves A[J,J] x = e_last (J = columns j <= i of row i, the diagonal last)
    and is x / sqrt(x_last).  Rows with more than max_len lower entries keep
    1/sqrt(a_ii) on the diagonal (the CUDA kernel's bound).  Returns G on the
    lower edges in CSR order (the order of lower_edges)."""
    row = np.asarray(row, np.int64)
    col = np.asarray(col, np.int64)
    A = sp.csr_matrix((np.asarray(val, np.float64), col, row), shape=(len(row) - 1, len(row) - 1))
    out = []
    for i in range(len(row) - 1):
        J = col[row[i]:row[i + 1]]
        J = J[J <= i]
        if len(J) > max_len:
            g = np.zeros(len(J))
            g[-1] = 1.0 / math.sqrt(A[i, i])
        else:
            B = A[J][:, J].toarray()
            e = np.zeros(len(J))
            e[-1] = 1.0
            x = np.linalg.solve(B, e)
            g = x / math.sqrt(x[-1])
        out.append(g)
    return np.concatenate(out) if out else np.zeros(0)


def probes(n, P, seed):
    """Rademacher probes: the same +-1 hash as the CUDA kernel k_fsai_probes."""
    i = np.arange(n, dtype=np.uint64)[:, None]
    p = np.arange(P, dtype=np.uint64)[None, :]
    with np.errstate(over="ignore"):
        h = (i * np.uint64(P) + p) ^ (np.uint64(seed) * np.uint64(0x9E3779B97F4A7C15))
        h ^= h >> np.uint64(33)
        h *= np.uint64(0xFF51AFD7ED558CCD)
        h ^= h >> np.uint64(33)
        h *= np.uint64(0xC4CEB9FE1A85EC53)
        h ^= h >> np.uint64(33)
    return np.where((h & np.uint64(1)) == 1, 1.0, -1.0)


class System:
    """One SPD system with everything the loss needs; base "ky" makes the
    network correct the Kolotilina-Yeremin G (ky_fsai) instead of Jacobi."""

    def __init__(self, row, col, val, xyz=None, base="none"):
        self.row = np.asarray(row, np.int64)
        self.col = np.asarray(col, np.int64)
        self.val = np.asarray(val, np.float64)
        self.n = len(self.row) - 1
        self.A = sp.csr_matrix((self.val, self.col, self.row), shape=(self.n, self.n))
        self.ky = ky_fsai(self.row, self.col, self.val) if base == "ky" else None
        (self.r, self.c, self.k, self.F, self.d, self.bnd, self.free, self.h) = features(row, col, val, xyz,
                                                                                          self.ky)

    def g(self, vec, rounding=True):
        out, _ = MLP(vec, rounding).forward(self.F)
        G, _ = g_values(out, self.r, self.c, self.val[self.k], self.d, self.free, self.ky)
        return G, out

    def loss(self, vec, Z, rounding=True, kind="residual"):
        G, _ = self.g(vec, rounding)
        return LOSSES[kind](self.A, g_matrix(self.n, self.r, self.c, G), self.r, self.c, Z)[0]

    def loss_and_grad(self, vec, Z, rounding=True, kind="residual"):
        mlp = MLP(vec, rounding)
        out, cache = mlp.forward(self.F)
        G, dGdo = g_values(out, self.r, self.c, self.val[self.k], self.d, self.free, self.ky)
        L, dG = LOSSES[kind](self.A, g_matrix(self.n, self.r, self.c, G), self.r, self.c, Z)
        return L, mlp.backward(cache, dG * dGdo), G


def init_params(seed, last_scale=0.0):
    """He-style initial weights; the last layer scaled by last_scale (0 gives
    G = D^-1/2, i.e. M = Jacobi)."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, shape in LAYOUT:
        if name.startswith("W"):
            p[name] = rng.standard_normal(shape) * math.sqrt(2.0 / shape[0])
        elif name == "w4":
            p[name] = rng.standard_normal(shape) * math.sqrt(1.0 / shape[0]) * last_scale
        else:
            p[name] = np.zeros(shape)
    return pack(p).astype(np.float32)
