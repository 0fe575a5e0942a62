"""Host-side mirror of the reference's solver entry, on the B200 path.

Names and meanings follow the reference's C++ host:
  SolverConfig{tau=1e-10, max_iters=0}           include/cg_common.hpp:52-55
  run_defaults.kTau / kMaxIters                  host/run_defaults.hpp:12-13
  CsrDataset.load(dir) and its checks            src/CsrDataset.hpp:19-67
  extract_jacobi_diag / build_jacobi_inverse     src/CsrDataset.hpp:92-116, host/pcg_common.hpp:42-54
  SolverStatus {converged, max_iter, breakdown}  host/pcg_common.hpp:16-33
  GoldenIterationTrace {alpha,beta,rz,rr,residual} src/CgSolverGolden.hpp:15-22
  result fields solution / iterations / final_rr / converged / status / residual_l2 /
  residual_rel / timing                          host/cuper_pcg_solver.hpp:62-73
  log_iteration "[iter NNN] alpha=..."           host/pcg_common.hpp:56-77
Tolerance semantics are the reference's by default (recurrence rr <= tau, absolute);
tau_mode=TAU_REL_TRUE asks for the FP64 true relative residual instead.

Every solve runs on the GPU through libxplus_b200.so.  Errors the reference throws as
std::runtime_error come back as XplusError with the same message.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import (XPLUS_F32, XPLUS_F64, XPLUS_BF16, XPLUS_F16, XPLUS_TAU_ABS_RR, XPLUS_TAU_REL_TRUE,
                   STATUS_NAMES, XplusError, check, lib, ptr)


class run_defaults:  # noqa: N801  (mirrors the reference namespace)
    kTau = 1.0e-10
    kMaxIters = 0
    kDeviceIndex = 0


kBreakdownEps = 1.0e-30
KERNEL_NAMES = {0: "pcg_persistent_kernel", 1: "pcg_resident_kernel", 2: "pcg_resident1_kernel",
                3: "pcg_gtg_kernel"}
kMaxN = 1024  # the reference multi-kernel cap; the GPU path has none


@dataclass
class SolverConfig:
    tau: float = run_defaults.kTau
    max_iters: int = run_defaults.kMaxIters


@dataclass
class IterationTrace:
    iteration: int
    alpha: float
    beta: float
    rz: float
    rr: float
    residual: float


@dataclass
class PcgResult:
    solution: np.ndarray
    iterations: int
    effective_max_iters: int
    final_rr: float
    status: str
    converged: bool
    residual_l2: float
    residual_rel: float
    iteration_trace: list = field(default_factory=list)
    replacements: int = 0
    kernel_ms: float = 0.0
    setup_ms: float = 0.0
    metrics: dict = field(default_factory=dict)


class CsrDataset:
    """The five-array CSR system of src/CsrDataset.hpp, loaded and validated natively."""

    def __init__(self, row_ptr, col_idx, values, b, x0):
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, dtype=np.int32)
        self.values = np.ascontiguousarray(values, dtype=np.float64)
        self.b = np.ascontiguousarray(b, dtype=np.float64)
        self.x0 = np.ascontiguousarray(x0, dtype=np.float64)

    @property
    def n(self) -> int:
        return len(self.row_ptr) - 1

    @property
    def nnz(self) -> int:
        return len(self.col_idx)

    @classmethod
    def load(cls, dataset_dir) -> "CsrDataset":
        d = str(Path(dataset_dir)).encode()
        n, nnz = C.c_int(), C.c_int()
        check(lib.xplus_dataset_load_text(d, C.byref(n), C.byref(nnz), None, None, None, None, None))
        rp = np.empty(n.value + 1, np.int32)
        ci = np.empty(nnz.value, np.int32)
        v = np.empty(nnz.value, np.float64)
        b = np.empty(n.value, np.float64)
        x0 = np.empty(n.value, np.float64)
        check(lib.xplus_dataset_load_text(d, C.byref(n), C.byref(nnz), ptr(rp), ptr(ci), ptr(v), ptr(b), ptr(x0)))
        return cls(rp, ci, v, b, x0)

    def save_binary(self, path) -> None:
        check(lib.xplus_dataset_save_binary(str(path).encode(), self.n, self.nnz, ptr(self.row_ptr),
                                            ptr(self.col_idx), ptr(self.values), ptr(self.b), ptr(self.x0)))

    @classmethod
    def load_binary(cls, path) -> "CsrDataset":
        p = str(path).encode()
        n, nnz = C.c_int(), C.c_int()
        check(lib.xplus_dataset_load_binary(p, C.byref(n), C.byref(nnz), None, None, None, None, None))
        rp = np.empty(n.value + 1, np.int32)
        ci = np.empty(nnz.value, np.int32)
        v = np.empty(nnz.value, np.float64)
        b = np.empty(n.value, np.float64)
        x0 = np.empty(n.value, np.float64)
        check(lib.xplus_dataset_load_binary(p, C.byref(n), C.byref(nnz), ptr(rp), ptr(ci), ptr(v), ptr(b), ptr(x0)))
        return cls(rp, ci, v, b, x0)

    def save_text(self, dataset_dir) -> None:
        """Writes the five text files in the reference's format (%.17g, space separated)."""
        d = Path(dataset_dir)
        d.mkdir(parents=True, exist_ok=True)
        for name, arr, fmt in (("row_ptr.txt", self.row_ptr, "%d"), ("col_idx.txt", self.col_idx, "%d"),
                               ("values.txt", self.values, "%.17g"), ("b.txt", self.b, "%.17g"),
                               ("x0.txt", self.x0, "%.17g")):
            (d / name).write_text(" ".join(fmt % v for v in arr.tolist()) + "\n")

    def extract_jacobi_diag(self) -> np.ndarray:
        diag = np.empty(self.n, np.float64)
        check(lib.xplus_jacobi_diag(self.n, ptr(self.row_ptr), ptr(self.col_idx), ptr(self.values), ptr(diag)))
        return diag


def build_jacobi_inverse(dataset: CsrDataset) -> np.ndarray:
    diag = dataset.extract_jacobi_diag()
    if np.any(np.abs(diag) <= kBreakdownEps):
        raise XplusError(_lib.XPLUS_ERR_DATA, "zero diagonal entry while building Jacobi inverse")
    return 1.0 / diag


def log_iteration(iteration: int, alpha: float, beta: float, rz: float, rr: float) -> str:
    """The "[iter NNN] ..." line of host/pcg_common.hpp:56-77."""
    return (f"[iter {iteration:03d}] alpha={alpha:.12e} beta={beta:.12e} rz={rz:.12e} "
            f"rr={rr:.12e} residual={math.sqrt(max(rr, 0.0)):.12e}")


_TYPES = {"f32": XPLUS_F32, "fp32": XPLUS_F32, "float32": XPLUS_F32, "bf16": XPLUS_BF16,
          "bfloat16": XPLUS_BF16, "f64": XPLUS_F64, "fp64": XPLUS_F64, "float64": XPLUS_F64,
          "f16": XPLUS_F16, "fp16": XPLUS_F16, "float16": XPLUS_F16}


def _type(t) -> int:
    return _TYPES[t] if isinstance(t, str) else int(t)


def _metrics_dict(m) -> dict:
    return dict(rz=m.rz, rr=m.rr, pap=m.pap, alpha=m.alpha, stagnated=bool(m.reserved[0]),
                device_ms=m.reserved[1], kernel=KERNEL_NAMES.get(int(m.reserved[2]), "unknown"),
                jacobi_fallback_at=int(m.reserved[3]) if int(m.reserved[2]) == 3 else -1)


class PcgSolver:
    """One SPD system resident on the GPU (xplus_pcg handle)."""

    def __init__(self, row_ptr, col_idx, values, *, values_dtype="f32", vector_dtype="f32",
                 sigma=256, chunk=4, keep_fp64=True, replace_every=0, replace_drop=1e-2,
                 block_threads=0, blocks_per_sm=0, barrier_timeout_s=2.0, device=0,
                 row_sum_form=True, index16=True, l2_persist=True, resident=True,
                 barriers_per_iter=1, restart_on_replace=-1, stagnation_gain=0.05, stagnation_window=8,
                 build_on_gpu=True, split_ratio=-1.0):
        self.row_ptr = np.ascontiguousarray(row_ptr, np.int32)
        self.col_idx = np.ascontiguousarray(col_idx, np.int32)
        self.values = np.ascontiguousarray(values, np.float64)
        self.n = len(self.row_ptr) - 1
        self.opts = _lib.default_opts(
            value_type=_type(values_dtype), vector_type=_type(vector_dtype), sigma=sigma, chunk=chunk,
            keep_fp64=int(keep_fp64), replace_every=replace_every, replace_drop=replace_drop,
            block_threads=block_threads, blocks_per_sm=blocks_per_sm,
            barrier_timeout_s=barrier_timeout_s, device=device, row_sum_form=int(row_sum_form), index16=int(index16),
            l2_persist=int(l2_persist), resident=int(resident), barriers_per_iter=int(barriers_per_iter),
            restart_on_replace=int(restart_on_replace), stagnation_gain=float(stagnation_gain),
            stagnation_window=int(stagnation_window), build_on_gpu=int(build_on_gpu),
            split_ratio=float(split_ratio))
        h = C.c_void_p()
        check(lib.xplus_pcg_create(ptr(self.row_ptr), ptr(self.col_idx), ptr(self.values), self.n,
                                   C.byref(self.opts), C.byref(h)))
        self._h = h

    @classmethod
    def from_dataset(cls, dataset: CsrDataset, **kw) -> "PcgSolver":
        return cls(dataset.row_ptr, dataset.col_idx, dataset.values, **kw)

    @property
    def handle(self):
        return self._h

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib.xplus_pcg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self) -> dict:
        vals = [C.c_int64() for _ in range(5)]
        check(lib.xplus_pcg_info(self._h, *[C.byref(v) for v in vals]))
        return dict(zip(("n", "n_pad", "nnz", "slots", "spmv_bytes"), (v.value for v in vals)))

    def solve(self, b, x0=None, *, tau=run_defaults.kTau, tau_mode=XPLUS_TAU_ABS_RR,
              max_iters=run_defaults.kMaxIters, trace=False) -> PcgResult:
        b = np.ascontiguousarray(b, np.float64)
        x = np.empty(self.n, np.float64)
        x0a = None if x0 is None else np.ascontiguousarray(x0, np.float64)
        eff = max_iters if max_iters > 0 else max(4 * self.n, 1000)
        hist = np.zeros(eff, np.float64) if trace else None
        iters = C.c_int()
        m = _lib.XplusMetrics()
        check(lib.xplus_pcg_solve(self._h, ptr(b), ptr(x0a), float(tau), int(tau_mode), int(max_iters),
                                  ptr(x), C.byref(iters), ptr(hist), eff if trace else 0, C.byref(m)))
        tr = []
        if trace and m.iterations > 0:
            rows = min(m.iterations, eff)
            t = np.empty(rows * 5, np.float64)
            check(lib.xplus_pcg_last_trace(self._h, ptr(t), rows))
            t = t.reshape(rows, 5)
            tr = [IterationTrace(k, *map(float, t[k])) for k in range(rows)]
        bnorm = float(np.linalg.norm(b))
        res_rel = m.true_rel_residual
        status = STATUS_NAMES.get(m.status, "unknown")
        return PcgResult(
            solution=x, iterations=m.iterations, effective_max_iters=eff, final_rr=m.rr,
            status=status, converged=(m.status == 0), residual_l2=res_rel * bnorm,
            residual_rel=res_rel, iteration_trace=tr, replacements=m.replacements,
            kernel_ms=m.kernel_ms, setup_ms=m.setup_ms, metrics=_metrics_dict(m))

    def solve_device(self, d_b, d_x, *, tau=1e-8, tau_mode=XPLUS_TAU_REL_TRUE, max_iters=0, stream=None) -> None:
        """Enqueues one solve on device-resident FP64 vectors (original row order; d_x holds
        x0 and receives x) on `stream` (a torch.cuda.Stream or raw handle; None: the
        solver's own) and returns without waiting.  last_metrics() waits and reports."""
        s = getattr(stream, "cuda_stream", stream)
        check(lib.xplus_pcg_solve_device(self._h, ptr(d_b), ptr(d_x), float(tau), int(tau_mode),
                                         int(max_iters), s))

    def phase_times(self) -> dict:
        """Phase clock of the last solve (ms summed over its iterations): block 0's four
        phases (xplus_pcg_last_phase_times) and the median over all CTAs of each phase
        (xplus_pcg_last_block_times)."""
        p = np.empty(4, np.float64)
        check(lib.xplus_pcg_last_phase_times(self._h, ptr(p)))
        nb = C.c_int()
        check(lib.xplus_pcg_last_block_times(self._h, None, 0, C.byref(nb)))
        blk = np.empty(4 * nb.value, np.float64)
        check(lib.xplus_pcg_last_block_times(self._h, ptr(blk), nb.value, C.byref(nb)))
        return {"block0_ms": p.tolist(), "median_ms": np.median(blk.reshape(-1, 4), axis=0).tolist()}

    def last_metrics(self) -> dict:
        """Outcome of the last solve (waits for it): status, iterations, replacements,
        true relative residual, kernel time and the kernel's own counters."""
        m = _lib.XplusMetrics()
        check(lib.xplus_pcg_last_metrics(self._h, C.byref(m)))
        out = _metrics_dict(m)
        out.update(status=STATUS_NAMES.get(m.status, "unknown"), converged=(m.status == 0),
                   iterations=m.iterations, replacements=m.replacements,
                   residual_rel=m.true_rel_residual, kernel_ms=m.kernel_ms)
        return out

    def set_gtg(self, g_low, fallback_iters: int = 0) -> None:
        """M^-1 = G^T G with G given on A's lower pattern (g_low order); None: Jacobi again."""
        g = None if g_low is None else np.ascontiguousarray(g_low, np.float64)
        check(lib.xplus_pcg_set_gtg(self._h, ptr(self.row_ptr), ptr(self.col_idx), ptr(g), int(fallback_iters)))

    def set_gnn(self, params=None, fallback_iters: int = 0, refine_sweeps: int = 4) -> float:
        """M^-1 = G^T G with G predicted on the GPU by the learned network (default: the
        shipped weights), refined by `refine_sweeps` Gauss-Seidel sweeps on each row's quadratic
        form and normalized to (G A G^T)_ii = 1.  Returns the inference time in ms."""
        from .learned import load_weights
        if params is None:
            params, _ = load_weights()
        p = np.ascontiguousarray(params, np.float32)
        ms = C.c_double()
        check(lib.xplus_pcg_set_gnn_ex(self._h, ptr(self.row_ptr), ptr(self.col_idx), ptr(self.values), ptr(p),
                                       int(fallback_iters), int(refine_sweeps), C.byref(ms)))
        return ms.value

    def scale_gtg(self) -> None:
        """Rescales the rows of the current G to (G A G^T)_ii = 1."""
        check(lib.xplus_pcg_scale_gtg(self._h, ptr(self.row_ptr), ptr(self.col_idx), ptr(self.values)))

    def get_gtg(self) -> np.ndarray:
        n = C.c_int64()
        check(lib.xplus_pcg_get_gtg(self._h, None, C.byref(n)))
        g = np.empty(n.value, np.float64)
        check(lib.xplus_pcg_get_gtg(self._h, ptr(g), C.byref(n)))
        return g

    def spmv(self, x) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float64)
        y = np.empty(self.n, np.float64)
        check(lib.xplus_pcg_spmv(self._h, ptr(x), ptr(y)))
        return y


def run_pcg(dataset: CsrDataset, config: SolverConfig = SolverConfig(), *, log=None, **opts) -> PcgResult:
    """Solve dataset with x0 and b from the dataset, the counterpart of
    run_cuper_pcg_solver(dataset, config, log) (host/cuper_pcg_solver.hpp:311)."""
    tau_mode = opts.pop("tau_mode", XPLUS_TAU_ABS_RR)
    solver = PcgSolver.from_dataset(dataset, **opts)
    try:
        res = solver.solve(dataset.b, dataset.x0, tau=config.tau, tau_mode=tau_mode,
                           max_iters=config.max_iters, trace=log is not None)
    finally:
        solver.close()
    if log is not None:
        log.write(f"[init] n={dataset.n} nnz={dataset.nnz} tau={config.tau:.12e} "
                  f"max_iters={res.effective_max_iters} dtype=b200-sell\n")
        for t in res.iteration_trace:
            log.write(log_iteration(t.iteration, t.alpha, t.beta, t.rz, t.rr) + "\n")
    return res


def device_count() -> int:
    return int(lib.xplus_device_count())
