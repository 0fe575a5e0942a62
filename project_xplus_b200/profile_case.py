"""A bounded run of the hot path for profilers (ncu): the 2D P1-FEM system of a given grid,
one warm-up solve and one profiled solve capped at a fixed number of iterations, then a
few standalone SELL SpMV launches.  Every kernel here is a product kernel.

  python -m project_xplus_b200.profile_case --grid 1108 --iters 100 --spmv 5
"""
from __future__ import annotations

import argparse
import ctypes as C

import numpy as np

from . import _lib
from . import generators as g
from .solver import PcgSolver


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--grid", type=int, default=1108)
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--spmv", type=int, default=5)
    ap.add_argument("--values", default="f32")
    ap.add_argument("--vectors", default="f32")
    ap.add_argument("--chunk", type=int, default=4)
    ap.add_argument("--dim3", type=int, default=0, help="use the 3D P1-FEM system with this grid side instead")
    ap.add_argument("--plain", action="store_true",
                    help="plain layout: values with the diagonal, int32 columns (no row-sum form)")
    a = ap.parse_args()
    d, _ = g.system_3d(a.dim3) if a.dim3 else g.system_2d_large(a.grid)
    extra = dict(row_sum_form=False, index16=False) if a.plain else {}
    s = PcgSolver.from_dataset(d, values_dtype=a.values, vector_dtype=a.vectors, chunk=a.chunk, **extra)
    for _ in range(2):
        r = s.solve(d.b, None, tau=1e-300, max_iters=a.iters)
    xs, ys = C.c_void_p(), C.c_void_p()
    _lib.check(_lib.lib.xplus_pcg_scratch_vectors(s.handle, C.byref(xs), C.byref(ys)))
    for _ in range(a.spmv):
        _lib.check(_lib.lib.xplus_pcg_spmv_device(s.handle, xs, ys, None))
    y = s.spmv(np.ones(d.n))
    print(f"n={d.n} nnz={d.nnz} iterations={r.iterations} kernel_ms={r.kernel_ms:.3f} "
          f"us/iter={1e3 * r.kernel_ms / max(1, r.iterations):.2f} info={s.info()} y0={y[0]:.6e}")
    s.close()


if __name__ == "__main__":
    main()
