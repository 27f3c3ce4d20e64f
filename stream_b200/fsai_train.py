"""Train the learned FSAI network on the GPU.

Training systems come from the pipeline itself: dam-break columns
(0.4 x 0.8 x 0.4, jittered lattice, alpha = 1.2 h) of n_min..n_max particles
(log-uniform), displaced by random Taylor-Green velocity fields over 1..20
Euler steps of dt = 0.005, remeshed by AlphaShape3D and assembled by
PoissonSystem (P1 Laplacian, free-surface Dirichlet rows, divergence
right-hand side).  `systems` of them are generated over the run and streamed
through a resident pool of `pool` systems (one replaced every few steps), so
device memory stays bounded.  Every Adam step takes the loss of one pool
system over 16 fresh Rademacher probes (or the mean over --batch systems),
through the library's forward/backward kernels (FsaiModel.train_step /
train_batch): --loss residual, sum_p ||G A G^T z_p - z_p||^2 / (16 n), or
--loss kaporin, log(t/n) - (2/n) sum_i log G_ii with t the probe estimate of
tr(G A G^T) (Kaporin's condition number, which the optimal FSAI minimises).
With --base ky the network learns a correction to each system's
Kolotilina-Yeremin G (zero output = that G) instead of to Jacobi.  The result
is written as a float32 vector of FsaiModel.PARAM_COUNT values (default: the
package's fsai_weights.npy, or fsai_weights_ky.npy with --base ky).

    python -m stream_b200.fsai_train --systems 2000 --steps 20000 --batch 4 --out stream_b200/fsai_weights.npy
    python -m stream_b200.fsai_train --base ky --systems 2000 --steps 20000 --batch 2
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import workloads

DT = 0.005


def displaced_column(n_target, rng):
    """Dam-break column of about n_target particles advected by a random
    Taylor-Green field for 1..20 Euler steps of DT (on the GPU)."""
    from .pfem import TaylorGreen, advect_taylor_green
    h = (0.4 * 0.8 * 0.4 / n_target) ** (1.0 / 3.0)
    pts, alpha = workloads.dambreak_column(h=h, seed=int(rng.integers(1 << 31)))
    x = advect_taylor_green(pts, TaylorGreen.random(rng), DT, int(rng.integers(1, 21)))
    return x.astype(np.float32), alpha


def divergence_modes(rng, count=8):
    k = rng.normal(size=(count, 3)) * 6.0
    amp = rng.normal(size=(count, 3))
    return np.concatenate([k, np.sum(amp * k, 1, keepdims=True), rng.uniform(0, 2 * math.pi, (count, 1))],
                          1).astype(np.float32)


def pipeline_system(n_target, rng):
    from .mesh import AlphaShape3D
    from .numerics import PoissonSystem
    pts, alpha = displaced_column(n_target, rng)
    mesh = AlphaShape3D()
    mesh.set_nodes(pts, alpha)
    mesh.compute()
    ps = PoissonSystem()
    ps.assemble(mesh, rhs="div", modes=divergence_modes(rng))
    return ps


def initial_params(seed):
    """He-initialised hidden layers, zero output layer (the untrained network is Jacobi)."""
    from .numerics import FsaiModel
    rng = np.random.default_rng(seed)
    shapes = [(16, 64), (64,), (64, 64), (64,), (64, 64), (64,), (64,), (1,)]
    parts = []
    for s in shapes:
        if len(s) == 2:
            parts.append(rng.standard_normal(s).reshape(-1) * math.sqrt(2.0 / s[0]))
        else:
            parts.append(np.zeros(s[0]))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == FsaiModel.PARAM_COUNT
    return p


def evaluate(model, n, seed, rtol=1e-8):
    import os
    from .numerics import FsaiModel, PoissonSystem
    rng = np.random.default_rng(seed)
    ps = pipeline_system(n, rng)
    out = {"n": ps.size()[0], "nnz": ps.size()[1]}
    _, r0 = ps.solve(method=PoissonSystem.FP64_JACOBI, rtol=rtol)
    out["jacobi_fp64"] = r0
    ps.set_fsai(FsaiModel(base=model.base))
    _, r1 = ps.solve(method=PoissonSystem.FSAI_MIXED, rtol=rtol)
    out["untrained_fsai_mixed"] = r1
    ps.set_fsai(model)
    _, r2 = ps.solve(method=PoissonSystem.FSAI_MIXED, rtol=rtol)
    out["trained_fsai_mixed"] = r2
    _, rk = ps.solve(method=PoissonSystem.KY_FSAI_MIXED, rtol=rtol)
    out["ky_fsai_mixed"] = rk
    if os.path.exists(FsaiModel.weights_path(model.base)):
        ps.set_fsai(FsaiModel.trained(model.base))
        _, r3 = ps.solve(method=PoissonSystem.FSAI_MIXED, rtol=rtol)
        out["shipped_fsai_mixed"] = r3
    ps.set_fsai(model)
    _, r2 = ps.solve(method=PoissonSystem.FSAI_MIXED, rtol=rtol)
    out["fsai_stats"] = ps.fsai_stats()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--systems", type=int, default=2000, help="systems generated over the run")
    ap.add_argument("--pool", type=int, default=64, help="systems resident at a time")
    ap.add_argument("--n-min", type=int, default=50_000)
    ap.add_argument("--n-max", type=int, default=500_000)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lr-min", type=float, default=5e-5)
    ap.add_argument("--clip", type=float, default=1.0)
    ap.add_argument("--batch", type=int, default=1, help="systems per Adam step (mean loss and gradient)")
    ap.add_argument("--loss", choices=["residual", "kaporin"], default="residual")
    ap.add_argument("--base", choices=["none", "ky"], default="none",
                    help="what the network corrects: Jacobi (none) or the Kolotilina-Yeremin G (ky)")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--init", default=None, help="start from these weights (.npy)")
    ap.add_argument("--eval-n", type=int, default=1_000_000)
    ap.add_argument("--out", default=None)
    ap.add_argument("--log", default=None, help="write the loss curve and evaluation as JSON here")
    a = ap.parse_args(argv)

    from .numerics import FsaiModel
    rng = np.random.default_rng(a.seed)

    def draw_n():
        return int(math.exp(rng.uniform(math.log(a.n_min), math.log(a.n_max))))

    t0 = time.time()
    pool = [pipeline_system(draw_n(), rng) for _ in range(min(a.pool, a.systems))]
    generated = len(pool)
    t_gen = time.time() - t0
    replace_every = max(1, a.steps // max(1, a.systems - generated))
    model = FsaiModel(np.load(a.init) if a.init else initial_params(a.seed), loss=a.loss, base=a.base)
    curve = []
    t1 = time.time()
    for step in range(a.steps):
        if step and step % replace_every == 0 and generated < a.systems:
            tg = time.time()
            pool[int(rng.integers(len(pool)))] = pipeline_system(draw_n(), rng)
            generated += 1
            t_gen += time.time() - tg
        lr = a.lr_min + 0.5 * (a.lr - a.lr_min) * (1 + math.cos(math.pi * step / max(1, a.steps)))
        if a.batch > 1:
            batch = [pool[int(i)] for i in rng.choice(len(pool), size=min(a.batch, len(pool)), replace=False)]
            loss = model.train_batch(batch, seed=int(rng.integers(1 << 62)), lr=lr, clip=a.clip)
        else:
            ps = pool[int(rng.integers(len(pool)))]
            loss = model.train_step(ps, seed=int(rng.integers(1 << 62)), lr=lr, clip=a.clip)
        if not math.isfinite(loss):
            raise RuntimeError(f"non-finite loss at step {step}")
        curve.append(loss)
    t_train = time.time() - t1 - (t_gen - (t1 - t0))
    params = model.get_params()
    out = a.out or FsaiModel.weights_path(a.base)
    np.save(out, params)
    summary = {
        "systems_generated": generated, "pool": len(pool), "n_range": [a.n_min, a.n_max], "steps": a.steps,
        "loss": a.loss, "base": a.base, "batch": a.batch,
        "generate_s": round(t_gen, 2), "train_s": round(t_train, 2),
        "loss_first100": float(np.mean(curve[:100])), "loss_last100": float(np.mean(curve[-100:])),
        "weights": out,
    }
    pool.clear()
    if a.eval_n:
        summary["eval"] = evaluate(model, a.eval_n, seed=10_000 + a.seed)
    print(json.dumps(summary))
    if a.log:
        with open(a.log, "w") as f:
            json.dump({**summary, "curve": curve[::10]}, f)


if __name__ == "__main__":
    main()
