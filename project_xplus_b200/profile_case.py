"""A bounded run of the hot path for profilers (ncu): the 2D P1-FEM system of a given grid (or
the 3D one), one warm-up solve and one profiled solve capped at a fixed number of iterations,
then a few standalone SELL SpMV launches.  Every kernel here is a product kernel.

  python -m project_xplus_b200.profile_case --grid 1108 --iters 100 --spmv 5
  python -m project_xplus_b200.profile_case --grid 1108 --iters 50 --spmv 0 --gtg fsai
  python -m project_xplus_b200.profile_case --batch 64 --iters 200 [--resident]
"""
from __future__ import annotations

import argparse
import ctypes as C

import numpy as np

from . import _lib
from . import generators as g
from .solver import PcgSolver


def batch_case(count: int, iters: int, resident: bool) -> None:
    """`count` systems of the batched workload's distribution, clusters of 8 x 512 threads
    (8 x 256 for the cluster-resident kernel), at most `iters` iterations per system, two
    launches."""
    from .batch import BatchSolver
    sides, sigmas = g.batch_sides(count, 45, 256, seed=3)
    systems = [g.fem2d(int(sd), sigma=float(sg), seed=1000 + k, x_seed=1000 + k)[0]
               for k, (sd, sg) in enumerate(zip(sides, sigmas))]
    s = BatchSolver([(d.row_ptr, d.col_idx, d.values) for d in systems])
    if resident:
        s.set_launch(8, 256)
        s.set_resident(True)
    else:
        s.set_launch(8, 512)
    b = np.concatenate([d.b for d in systems])
    for _ in range(2):
        r = s.solve(b, tau=1e-8, max_iters=iters)
    print(f"batch systems={count} kernel_ms={r['kernel_ms']:.3f} iterations={int(r['iterations'].sum())}")
    s.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=1108)
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--spmv", type=int, default=5)
    ap.add_argument("--values", default="f32")
    ap.add_argument("--vectors", default="f32")
    ap.add_argument("--chunk", type=int, default=4)
    ap.add_argument("--sigma", type=int, default=256, help="SELL sort window")
    ap.add_argument("--dim3", type=int, default=0, help="use the 3D P1-FEM system with this grid side instead")
    ap.add_argument("--plain", action="store_true",
                    help="plain layout: values with the diagonal, int32 columns (no row-sum form)")
    ap.add_argument("--gtg", choices=["fsai", "learned"], help="solve with M^-1 = G^T G (FSAI or learned G)")
    ap.add_argument("--batch", type=int, default=0, help="run the batched solver on this many systems instead")
    ap.add_argument("--resident", action="store_true", help="batched solver: the cluster-resident kernel")
    a = ap.parse_args()
    if a.batch:
        batch_case(a.batch, a.iters, a.resident)
        return
    d, _ = g.system_3d(a.dim3) if a.dim3 else g.system_2d_large(a.grid)
    extra = dict(row_sum_form=False, index16=False) if a.plain else {}
    s = PcgSolver.from_dataset(d, values_dtype=a.values, vector_dtype=a.vectors, chunk=a.chunk, sigma=a.sigma, **extra)
    if a.gtg == "fsai":
        from .learned import fsai_lower
        s.set_gtg(fsai_lower(d.row_ptr, d.col_idx, d.values))
    elif a.gtg == "learned":
        s.set_gnn()
    for _ in range(2):
        r = s.solve(d.b, None, tau=1e-300, max_iters=a.iters)
    xs, ys = C.c_void_p(), C.c_void_p()
    _lib.check(_lib.lib.xplus_pcg_scratch_vectors(s.handle, C.byref(xs), C.byref(ys)))
    for _ in range(a.spmv):
        _lib.check(_lib.lib.xplus_pcg_spmv_device(s.handle, xs, ys, None))
    y = s.spmv(np.ones(d.n))
    ph = s.phase_times()
    per_it = [round(1e3 * v / max(1, r.iterations), 2) for v in ph["median_ms"]]
    print(f"n={d.n} nnz={d.nnz} iterations={r.iterations} kernel_ms={r.kernel_ms:.3f} kernel={r.metrics['kernel']} "
          f"us/iter={1e3 * r.kernel_ms / max(1, r.iterations):.2f} phase_us/iter(median CTA)={per_it} "
          f"info={s.info()} y0={y[0]:.6e}")
    s.close()


if __name__ == "__main__":
    main()
