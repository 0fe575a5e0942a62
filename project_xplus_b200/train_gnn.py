"""Trains the learned G^T G preconditioner on the GPU and writes its weights.

Training systems come from the project's generators: 2D P1-FEM (jittered triangles) and
3D P1-FEM (Kuhn tetrahedra) stiffness matrices with log-normal conductivity sigma drawn
from [0.5, 2.5], each randomly permuted and then reverse Cuthill-McKee ordered (the order the
solver is benchmarked in).  Every step is one system, K = 8 probe vectors, Adam with a
cosine-decayed learning rate; forward, backward and Adam are the library's CUDA kernels.

  python -m project_xplus_b200.train_gnn --systems 256 --steps 20000 --nmin 16000 --nmax 256000
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np

from . import generators as gen
from .learned import DEFAULT_WEIGHTS, GnnTrainer, init_params, save_weights


def training_systems(count: int, nmin: int, nmax: int, seed: int):
    """`count` systems, half 2D and half 3D, n log-uniform in [nmin, nmax]."""
    rng = np.random.default_rng(seed)
    out, desc = [], []
    for k in range(count):
        n_target = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        sigma = float(math.exp(rng.uniform(math.log(0.5), math.log(2.5))))
        s = 10_000 + seed * 100_000 + k
        if k % 2 == 0:
            side = max(8, int(round(math.sqrt(n_target))))
            d, _ = gen.fem2d(side, sigma=sigma, jitter=0.3, seed=s, perm_seed=s, rcm=True, x_seed=s)
            desc.append(("2d", side, sigma))
        else:
            side = max(4, int(round(n_target ** (1.0 / 3.0))))
            d, _ = gen.fem3d(side, sigma=sigma, jitter=0.25, seed=s, perm_seed=s, rcm=True, x_seed=s)
            desc.append(("3d", side, sigma))
        out.append(d)
    return out, desc


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=256)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--nmin", type=int, default=16000)
    ap.add_argument("--nmax", type=int, default=256000)
    ap.add_argument("--probes", type=int, default=8)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    a = ap.parse_args()
    t0 = time.time()
    systems, desc = training_systems(a.systems, a.nmin, a.nmax, a.seed)
    t_gen = time.time() - t0
    t1 = time.time()
    tr = GnnTrainer([(d.row_ptr, d.col_idx, d.values) for d in systems], probes=a.probes, params=init_params(0))
    t_up = time.time() - t1
    t2 = time.time()
    losses = tr.train(a.steps, lr=a.lr, lr_final=a.lr_final, seed=a.seed)
    t_train = time.time() - t2
    params = tr.params()
    tr.close()
    w = max(1, a.steps // 20)
    curve = [float(losses[i:i + w].mean()) for i in range(0, a.steps, w)]
    meta = {"systems": a.systems, "steps": a.steps, "probes": a.probes, "n_range": [a.nmin, a.nmax],
            "sum_n": int(sum(d.n for d in systems)), "lr": a.lr, "lr_final": a.lr_final, "seed": a.seed,
            "generator": "fem2d (jitter 0.3) / fem3d (jitter 0.25), sigma log-uniform [0.5, 2.5], random perm + RCM",
            "loss_first": float(losses[:w].mean()), "loss_last": float(losses[-w:].mean()), "loss_curve": curve,
            "seconds": {"generate": round(t_gen, 1), "upload": round(t_up, 1), "train": round(t_train, 1)}}
    save_weights(a.out, params, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
