"""Generates the committed golden fixtures by running the REFERENCE ITSELF, compiled from
its own sources (oracle/_ref/libxplus_ref.so, built by oracle/Makefile from the reference
tree), on small seeded systems.  Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py

Each fixture stores the input system and the reference's outputs:
  golden_<name>.npz : row_ptr col_idx values b x0, tau, max_iters,
                      golden_x, golden_trace[k,5], golden_iterations,
                      mk_x, mk_trace, mk_status, mk_iterations           (multi-kernel solver)
                      ctl_x, ctl_metrics, ctl_status, ctl_iterations    (control kernel, packed FP32 SpMV)
                      cuper_spmv_y (cuper_style_spmv of x_true)
                      pack_ptr, pack_words, pack_channel_words          (16-channel packer)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle import oracle as O  # noqa: E402
from project_xplus_b200 import generators as g  # noqa: E402

OUT = Path(__file__).resolve().parent


def cases():
    # (name, dataset, x_true, tau, max_iters)
    d0, x0 = g.fem2d(32, sigma=1.0, jitter=0.3, seed=0, x_seed=0)
    yield "fem2d_g32", d0, x0, 1e-10, 0
    d1, x1 = g.fem2d(20, sigma=2.0, jitter=0.3, seed=7, perm_seed=1, rcm=True, x_seed=0)
    yield "fem2d_g20_rcm", d1, x1, 1e-12, 0
    d2, x2 = g.fem3d(8, sigma=1.5, jitter=0.25, seed=0, x_seed=0)
    yield "fem3d_g8", d2, x2, 1e-12, 0
    # max-iteration stop: same system as fem2d_g32, cut at 20 iterations
    yield "fem2d_g32_maxit20", d0, x0, 1e-30, 20
    # non-zero x0 (a smooth start vector) on a 12x12 system
    d3, x3 = g.fem2d(12, sigma=0.5, jitter=0.2, seed=5, x_seed=2)
    d3.x0 = np.cos(0.3 * np.arange(d3.n))
    yield "fem2d_g12_x0", d3, x3, 1e-14, 0


def main():
    if O.reflib() is None:
        raise SystemExit("oracle/_ref/libxplus_ref.so missing: run `make -C oracle ref` with the reference tree")
    for name, d, xt, tau, mi in cases():
        gr = O.golden(d, tau, mi, use_ref=True)
        rec = dict(row_ptr=d.row_ptr, col_idx=d.col_idx, values=d.values, b=d.b, x0=d.x0,
                   x_true=xt, tau=tau, max_iters=mi,
                   golden_x=gr["x"], golden_trace=gr["trace"], golden_iterations=gr["iterations"],
                   golden_final_rr=gr["final_rr"])
        if d.n <= 1024:
            mk = O.multi_kernel(d, tau, mi, use_ref=True)
            rec.update(mk_x=mk["x"], mk_trace=mk["trace"], mk_status=mk["status"],
                       mk_iterations=mk["iterations"], mk_residual_l2=mk["residual_l2"])
        ctl = O.control_ref(d, tau, mi)
        rec.update(ctl_x=ctl["x"], ctl_metrics=ctl["metrics"], ctl_status=ctl["status"],
                   ctl_iterations=ctl["iterations"])
        rec["cuper_spmv_y"] = O.cuper_spmv(d, xt, use_ref=True)
        pk = O.cuper_pack_ref(d)
        rec.update(pack_ptr=pk["ptr"], pack_words=pk["words"], pack_channel_words=pk["channel_words"],
                   pack_batch_count=pk["batch_count"])
        np.savez_compressed(OUT / f"golden_{name}.npz", **rec)
        print(name, d.n, d.nnz, "golden it", gr["iterations"], "control it", ctl["iterations"])


if __name__ == "__main__":
    main()
