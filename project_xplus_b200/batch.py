"""Batched Jacobi-PCG: many independent SPD systems in one persistent launch (xplus_batch_*).

The reference runs one system per launch (host/cuper_control_xrt_host.cpp:205-272); a
caller with many systems loops over datasets.  BatchSolver keeps every system resident
and solves all of them with one launch of thread-block clusters fed by a device work queue.

Across GPUs the systems shard with no collective: `shard_systems` splits them over ranks
by estimated work (longest-processing-time first), and each rank runs its own BatchSolver.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import XPLUS_TAU_REL_TRUE, check, lib, ptr
from .solver import STATUS_NAMES, _type


def system_work(n: int, nnz: int) -> float:
    """Work estimate of one solve: nnz per iteration x iterations ~ sqrt(n) on these grids."""
    return float(nnz) * math.sqrt(float(n))


def shard_systems(works, world: int, rank: int) -> list[int]:
    """Indices of the systems rank `rank` of `world` solves: greedy longest-processing-time
    assignment (heaviest system first, to the least-loaded rank; ties to the lower rank), so
    every rank computes the same partition without communicating."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    order = sorted(range(len(works)), key=lambda k: (-works[k], k))
    load = [0.0] * world
    owner = [0] * len(works)
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[k] = r
        load[r] += works[k]
    return [k for k in range(len(works)) if owner[k] == rank]


class BatchSolver:
    """A batch of CSR systems resident on one GPU (xplus_batch handle)."""

    def __init__(self, systems, *, values_dtype="f32", sigma=256, chunk=4, index16=True,
                 replace_drop=1e-2, replace_every=0, restart_on_replace=-1, stagnation_gain=0.05,
                 stagnation_window=8, split_ratio=-1.0, device=0):
        self.systems = [(np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                         np.ascontiguousarray(v, np.float64)) for rp, ci, v in systems]
        k = len(self.systems)
        if k == 0:
            raise ValueError("empty batch")
        self.ns = np.array([len(rp) - 1 for rp, _, _ in self.systems], np.int32)
        self.offsets = np.concatenate([[0], np.cumsum(self.ns.astype(np.int64))])
        self.opts = _lib.default_opts(value_type=_type(values_dtype), sigma=sigma, chunk=chunk,
                                      index16=int(index16), replace_drop=replace_drop,
                                      replace_every=replace_every, restart_on_replace=restart_on_replace,
                                      stagnation_gain=stagnation_gain, stagnation_window=stagnation_window,
                                      split_ratio=float(split_ratio), device=device)
        rps = (C.c_void_p * k)(*[ptr(s[0]) for s in self.systems])
        cis = (C.c_void_p * k)(*[ptr(s[1]) for s in self.systems])
        vs = (C.c_void_p * k)(*[ptr(s[2]) for s in self.systems])
        h = C.c_void_p()
        check(lib.xplus_batch_create(k, rps, cis, vs, ptr(self.ns), C.byref(self.opts), C.byref(h)))
        self._h = h

    @property
    def nsys(self) -> int:
        return len(self.systems)

    @property
    def total_n(self) -> int:
        return int(self.offsets[-1])

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib.xplus_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        n, nnz, sp = C.c_int64(), C.c_int64(), C.c_int64()
        cl, tpb, grid = C.c_int(), C.c_int(), C.c_int()
        check(lib.xplus_batch_info(self._h, C.byref(n), C.byref(nnz), C.byref(cl), C.byref(tpb), C.byref(grid),
                                   C.byref(sp)))
        return dict(total_n=n.value, total_nnz=nnz.value, cluster=cl.value, block_threads=tpb.value,
                    grid=grid.value, spmv_bytes=sp.value, split_lane=self.split_lane(), resident=self.resident())

    def set_resident(self, on: bool = True) -> None:
        """Both launches on the cluster-resident kernel (vectors and the search direction's
        window in shared memory, one cluster barrier per iteration), or back to the
        global-memory kernel.  Raises when a system does not fit its launch's cluster size."""
        check(lib.xplus_batch_set_resident(self._h, 1 if on else 0))

    def resident(self) -> dict:
        on, sm, sm2 = C.c_int(), C.c_int(), C.c_int()
        check(lib.xplus_batch_resident_info(self._h, C.byref(on), C.byref(sm), C.byref(sm2)))
        return dict(on=bool(on.value), smem=sm.value, smem_split=sm2.value)

    def set_stage_matrix(self, on: bool = True) -> None:
        """Resident launches widened to the most shared memory that keeps their occupancy, and
        each band's matrix copied there when it fits (on by default; results are the same bit
        for bit either way)."""
        check(lib.xplus_batch_set_stage_matrix(self._h, 1 if on else 0))

    def staged(self) -> dict:
        """Matrix staging: on, and over the last resident solve the systems whose every CTA
        staged its band's matrix (all) or only some CTAs did (some)."""
        on, al, so = C.c_int(), C.c_int(), C.c_int()
        check(lib.xplus_batch_staged_info(self._h, C.byref(on), C.byref(al), C.byref(so)))
        return dict(on=bool(on.value), all=al.value, some=so.value)

    def set_split_lane(self, count: int, cluster: int = 16, block_threads: int = 512) -> None:
        """The `count` largest systems in a concurrent launch of their own (0: none)."""
        check(lib.xplus_batch_set_split(self._h, int(count), int(cluster), int(block_threads)))

    def split_lane(self) -> dict:
        k, cl, tpb, grid = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        check(lib.xplus_batch_split_info(self._h, C.byref(k), C.byref(cl), C.byref(tpb), C.byref(grid)))
        return dict(count=k.value, cluster=cl.value, block_threads=tpb.value, grid=grid.value)

    def set_launch(self, cluster: int, block_threads: int) -> None:
        check(lib.xplus_batch_set_launch(self._h, int(cluster), int(block_threads)))

    def autotune(self, iters: int = 0, tau: float = 1e-8) -> dict:
        """Kernel (global-memory or cluster-resident), launch shape and the lane of the largest
        systems: fixed `iters` iterations per system, or (iters=0) full solves to tau."""
        cl, tpb, ms = C.c_int(), C.c_int(), C.c_double()
        check(lib.xplus_batch_autotune(self._h, int(iters), float(tau), C.byref(cl), C.byref(tpb), C.byref(ms)))
        return dict(cluster=cl.value, block_threads=tpb.value, ms=ms.value, split_lane=self.split_lane(),
                    resident=self.resident())

    def split(self, x) -> list[np.ndarray]:
        return [x[self.offsets[k]:self.offsets[k + 1]] for k in range(self.nsys)]

    def solve(self, b, x0=None, *, tau=1e-8, tau_mode=XPLUS_TAU_REL_TRUE, max_iters=0) -> dict:
        b = np.ascontiguousarray(b, np.float64)
        if b.shape != (self.total_n,):
            raise ValueError("b must hold every system's right-hand side, concatenated")
        x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        x = np.empty(self.total_n, np.float64)
        check(lib.xplus_batch_solve(self._h, ptr(b), ptr(x0a), float(tau), int(tau_mode), int(max_iters), ptr(x)))
        r = self.results()
        r["x"] = x
        return r

    def solve_device(self, d_b, d_x, *, tau=1e-8, tau_mode=XPLUS_TAU_REL_TRUE, max_iters=0, stream=None) -> None:
        """Enqueues the solve (one CUDA graph) on `stream` (a torch.cuda.Stream or raw handle)."""
        s = getattr(stream, "cuda_stream", stream)
        check(lib.xplus_batch_solve_device(self._h, ptr(d_b), ptr(d_x), float(tau), int(tau_mode),
                                           int(max_iters), s))

    def results(self) -> dict:
        k = self.nsys
        st = np.empty(k, np.int32)
        it = np.empty(k, np.int32)
        rp = np.empty(k, np.int32)
        tr = np.empty(k, np.float64)
        ms = np.empty(k, np.float64)
        kms = C.c_double()
        check(lib.xplus_batch_results(self._h, ptr(st), ptr(it), ptr(rp), ptr(tr), ptr(ms), C.byref(kms)))
        return dict(status=st, iterations=it, replacements=rp, true_rel=tr, system_ms=ms, kernel_ms=kms.value,
                    status_names=[STATUS_NAMES.get(int(s), "unknown") for s in st])


def autotune_build(systems, b, *, sigmas=(32, 256, 1024), chunks=(2, 4), iters=0, tau=1e-8, values_dtype="f32",
                   **kw) -> tuple[BatchSolver, dict]:
    """The batch autotuner: every (sigma, chunk) SELL layout is built, each one's launch shape
    is tuned by xplus_batch_autotune (full solves to `tau`, or `iters` fixed iterations), and
    the fastest layout is kept.  Slice height stays 32 (one warp lane per row).  Returns the chosen solver and a
    table of what was timed.  `b` is unused by the timing (the tuner solves b = 1) and kept so
    a caller can solve right away."""
    best, table = None, []
    for sg in sigmas:
        for ch in chunks:
            s = BatchSolver(systems, values_dtype=values_dtype, sigma=sg, chunk=ch, **kw)
            t = s.autotune(iters, tau)
            table.append(dict(sigma=sg, chunk=ch, **t))
            if best is None or t["ms"] < best[1]["ms"]:
                if best is not None:
                    best[0].close()
                best = (s, dict(sigma=sg, chunk=ch, **t))
            else:
                s.close()
    best[1]["table"] = table
    return best[0], best[1]
