"""Trains the learned G^T G preconditioner on the GPU and writes its weights.

Training systems come from the project's generators: 2D P1-FEM (jittered triangles) and
3D P1-FEM (Kuhn tetrahedra) stiffness matrices with log-normal conductivity sigma drawn
from [0.5, 2.5], n log-uniform in [nmin, nmax], each randomly permuted and then reverse
Cuthill-McKee ordered (the order the solver is benchmarked in).  Every step is one system,
Adam with a cosine-decayed learning rate over all steps; forward, backward and Adam are the
library's CUDA kernels.  The default loss is the row-normalized Kaporin loss
(1/n) sum_i [log (G A G^T)_ii - 2 log Ghat_ii].

The systems are generated on the host's threads in chunks of --chunk systems; each chunk is
resident on the GPU for its share of the steps (steps x chunk / systems), so a set larger
than the device's memory trains under one schedule.

  python -m project_xplus_b200.train_gnn --systems 4096 --steps 20000 --nmin 16000 --nmax 256000
"""
from __future__ import annotations

import argparse
import json
import math
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import generators as gen
from .learned import DEFAULT_WEIGHTS, GnnTrainer, init_params, save_weights


def system_specs(count: int, nmin: int, nmax: int, seed: int):
    """(kind, side, sigma, seed) of `count` systems, alternating 2D and 3D, n log-uniform in
    [nmin, nmax], sigma log-uniform in [0.5, 2.5]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n_target = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        sigma = float(math.exp(rng.uniform(math.log(0.5), math.log(2.5))))
        s = 10_000 + seed * 100_000 + k
        if k % 2 == 0:
            out.append(("2d", max(8, int(round(math.sqrt(n_target)))), sigma, s))
        else:
            out.append(("3d", max(4, int(round(n_target ** (1.0 / 3.0)))), sigma, s))
    return out


def make_system(spec):
    kind, side, sigma, s = spec
    if kind == "2d":
        d, _ = gen.fem2d(side, sigma=sigma, jitter=0.3, seed=s, perm_seed=s, rcm=True, x_seed=s)
    else:
        d, _ = gen.fem3d(side, sigma=sigma, jitter=0.25, seed=s, perm_seed=s, rcm=True, x_seed=s)
    return d


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--systems", type=int, default=4096)
    ap.add_argument("--chunk", type=int, default=512, help="systems resident on the GPU at a time")
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--nmin", type=int, default=16000)
    ap.add_argument("--nmax", type=int, default=256000)
    ap.add_argument("--loss", default="kaporin", choices=["kaporin", "probe"])
    ap.add_argument("--probes", type=int, default=8)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--lr-final", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--threads", type=int, default=16)
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    a = ap.parse_args()
    specs = system_specs(a.systems, a.nmin, a.nmax, a.seed)
    chunks = [specs[i:i + a.chunk] for i in range(0, len(specs), a.chunk)]
    # steps of each chunk in proportion to its systems, summing to a.steps
    bounds = [round(a.steps * sum(len(c) for c in chunks[:k]) / len(specs)) for k in range(len(chunks) + 1)]
    t_gen = t_up = t_train = 0.0
    tr = None
    losses = []
    sum_n = 0
    pool = ThreadPoolExecutor(a.threads)
    nxt = pool.map(make_system, chunks[0])
    for k, chunk in enumerate(chunks):
        t0 = time.time()
        systems = list(nxt)
        t_gen += time.time() - t0
        sum_n += sum(d.n for d in systems)
        t1 = time.time()
        csr = [(d.row_ptr, d.col_idx, d.values) for d in systems]
        if tr is None:
            tr = GnnTrainer(csr, probes=a.probes, params=init_params(0), loss=a.loss)
        else:
            tr.load(csr)
        del systems, csr
        if k + 1 < len(chunks):
            nxt = pool.map(make_system, chunks[k + 1])  # generated while this chunk trains
        t_up += time.time() - t1
        t2 = time.time()
        steps = bounds[k + 1] - bounds[k]
        if steps > 0:
            losses.append(tr.train(steps, lr=a.lr, lr_final=a.lr_final, seed=a.seed, first_step=bounds[k],
                                   total_steps=a.steps))
        t_train += time.time() - t2
        print(f"chunk {k + 1}/{len(chunks)}: {len(chunk)} systems, steps {bounds[k]}..{bounds[k + 1]}, "
              f"loss {losses[-1][-min(50, steps):].mean() if steps else float('nan'):.5f}", flush=True)
    pool.shutdown()
    losses = np.concatenate(losses)
    params = tr.params()
    tr.close()
    w = max(1, a.steps // 20)
    curve = [float(losses[i:i + w].mean()) for i in range(0, a.steps, w)]
    meta = {"systems": a.systems, "chunk": a.chunk, "steps": a.steps, "loss": a.loss, "probes": a.probes,
            "n_range": [a.nmin, a.nmax], "sum_n": int(sum_n), "lr": a.lr, "lr_final": a.lr_final, "seed": a.seed,
            "generator": "fem2d (jitter 0.3) / fem3d (jitter 0.25), sigma log-uniform [0.5, 2.5], random perm + RCM",
            "loss_first": float(losses[:w].mean()), "loss_last": float(losses[-w:].mean()), "loss_curve": curve,
            "seconds": {"generate_wait": round(t_gen, 1), "upload": round(t_up, 1), "train": round(t_train, 1)}}
    save_weights(a.out, params, meta)
    print(json.dumps(meta))


if __name__ == "__main__":
    main()
