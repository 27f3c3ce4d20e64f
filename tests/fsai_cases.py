"""Small SPD systems for the learned-FSAI tests.

grid_system: a 3-D 7-point stencil on an m^3 jittered grid with random
symmetric weights, a Dirichlet face (identity rows, eliminated columns kept as
explicit zeros, as the P1 assembly writes them) and a positive shift, so that
the boundary-fraction and explicit-zero cases of the features all occur.
"""
import numpy as np


def grid_system(m=5, seed=0, shift=0.3):
    rng = np.random.default_rng(seed)
    n = m ** 3
    idx = np.arange(n).reshape(m, m, m)
    xyz = np.stack(np.meshgrid(*[np.arange(m)] * 3, indexing="ij"), -1).reshape(-1, 3) / (m - 1)
    xyz = xyz + rng.uniform(-0.02, 0.02, xyz.shape)
    dirichlet = np.zeros(n, bool)
    dirichlet[idx[:, :, m - 1].ravel()] = True
    weight = {}
    nbrs = [[] for _ in range(n)]
    for i in range(n):
        a, b, c = np.unravel_index(i, (m, m, m))
        for da, db, dc in [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]:
            aa, bb, cc = a + da, b + db, c + dc
            if 0 <= aa < m and 0 <= bb < m and 0 <= cc < m:
                j = int(idx[aa, bb, cc])
                nbrs[i].append(j)
                key = (min(i, j), max(i, j))
                if key not in weight:
                    weight[key] = -(0.5 + rng.random())
    row, col, val = [0], [], []
    for i in range(n):
        cols = sorted(nbrs[i] + [i])
        diag = shift + sum(-weight[(min(i, j), max(i, j))] for j in nbrs[i])
        for j in cols:
            col.append(j)
            if j == i:
                val.append(1.0 if dirichlet[i] else diag)
            else:
                val.append(0.0 if (dirichlet[i] or dirichlet[j]) else weight[(min(i, j), max(i, j))])
        row.append(len(col))
    return np.array(row, np.uint32), np.array(col, np.uint32), np.array(val, np.float64), xyz
