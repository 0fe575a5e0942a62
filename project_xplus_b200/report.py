"""Solve reports in the reference's formats, and a command-line solve.

The text and JSON reports keep the sections, keys and number formats of the reference's
report writer (archived/host/report_io.hpp:83-171 text, :173-282 JSON), so tools that read
the reference's reports read these.  The console lines follow its host programs:
  [done] iter=... residual_abs=... residual_rel=... status=...   (archived/host/cuper_pcg_main.cpp:104)
  [check] cpu_residual_abs=... b200_residual_abs=... max_abs_diff=... max_rel_diff=... diff_tol=...
  [timing-ms] setup=... solve=... kernel=... iterations=... us_per_iteration=...

  python -m project_xplus_b200.report DATASET_DIR [--tau T] [--max-iters K] [--rel]
         [--text-report PATH] [--json-report PATH] [--x-ref PATH]
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np


@dataclass
class ReportInputs:
    dataset_dir: str
    n: int
    nnz: int
    effective_max_iters: int
    tau: float
    device_index: int
    pass_: bool
    converged: bool
    breakdown: bool
    iterations: int
    final_rr: float
    residual_l2: float
    residual_rel: float
    max_abs_diff: float
    golden_residual_l2: float
    total_ms: float
    host_setup_ms: float
    h2d_ms: float
    kernel_ms: float
    d2h_ms: float
    verify_ms: float
    traces: list = field(default_factory=list)   # IterationTrace-like objects
    pcg_control_calls: int = 1


def _status(r: ReportInputs) -> str:
    return "breakdown" if r.breakdown else ("converged" if r.converged else "max_iter")


def _e(v: float) -> str:
    """std::scientific with precision 12."""
    return f"{v:.12e}"


def _f(v: float) -> str:
    """std::fixed with precision 3."""
    return f"{v:.3f}"


def text_report(r: ReportInputs) -> str:
    """The text report: [Problem], [Accuracy], [Host Timing ms], [Kernel Timing ms]."""
    avg = r.kernel_ms / r.pcg_control_calls if r.pcg_control_calls > 0 else 0.0
    lines = [
        "[Problem]",
        f"dataset            : {r.dataset_dir}",
        f"n / nnz            : {r.n} / {r.nnz}",
        f"max_iters          : {r.effective_max_iters}",
        f"tau                : {_e(r.tau)}",
        f"device_index       : {r.device_index}",
        "",
        "[Accuracy]",
        f"pass               : {'yes' if r.pass_ else 'no'}",
        f"converged          : {'yes' if r.converged else 'no'}",
        f"status             : {_status(r)}",
        f"iterations         : {r.iterations}",
        f"final_rr           : {_e(r.final_rr)}",
        f"final_residual     : {_e(r.residual_l2)}",
        f"residual_rel       : {_e(r.residual_rel)}",
        f"max_abs_diff       : {_e(r.max_abs_diff)}",
        f"golden_residual    : {_e(r.golden_residual_l2)}",
        "",
        "[Host Timing ms]",
        f"total              : {_f(r.total_ms)}",
        f"host_setup         : {_f(r.host_setup_ms)}",
        f"buffer_h2d         : {_f(r.h2d_ms)}",
        f"kernel_total       : {_f(r.kernel_ms)}",
        f"buffer_d2h         : {_f(r.d2h_ms)}",
        f"verify             : {_f(r.verify_ms)}",
        "",
        "[Kernel Timing ms]",
        f"pcg_control_total  : {_f(r.kernel_ms)}",
        f"pcg_control_avg    : {_f(avg)}",
        "split_timing_note  : not available for single pcg_control_kernel runs",
    ]
    for name in ("spmv", "init", "dot", "update_xrz", "update_p"):
        lines.append(f"{name + '_total':<19}: {_f(0.0)}")
        lines.append(f"{name + '_avg':<19}: {_f(0.0)}")
    return "\n".join(lines) + "\n"


def json_report(r: ReportInputs) -> dict:
    """The JSON report as a dict with the reference's keys (dataset, result, host_timing_ms,
    kernel_timing_ms, trace_metadata, iterations_trace).  The trace here is the GPU solve's own
    per-iteration record, not a CPU re-run."""
    calls = r.pcg_control_calls
    kt = {"pcg_control_total": r.kernel_ms, "pcg_control_avg": r.kernel_ms / calls if calls > 0 else 0.0,
          "pcg_control_calls": calls}
    for name in ("spmv", "init", "dot", "update_xrz", "update_p"):
        kt[f"{name}_total"] = 0.0
        kt[f"{name}_avg"] = 0.0
        kt[f"{name}_calls"] = 0
    kt["split_timing_available"] = False
    kt["timing_model"] = "single_control_kernel"
    return {
        "dataset": {"path": r.dataset_dir, "xclbin": "", "n": r.n, "nnz": r.nnz, "max_iters": r.effective_max_iters,
                    "tau": r.tau, "device_index": r.device_index},
        "result": {"pass": r.pass_, "converged": r.converged, "status": _status(r), "iterations": r.iterations,
                   "final_rr": r.final_rr, "final_residual_norm": r.residual_l2, "residual_rel": r.residual_rel,
                   "solution_max_abs_diff": r.max_abs_diff, "golden_residual_norm": r.golden_residual_l2},
        "host_timing_ms": {"total": r.total_ms, "host_setup": r.host_setup_ms, "buffer_h2d": r.h2d_ms,
                           "kernel_total": r.kernel_ms, "buffer_d2h": r.d2h_ms, "verify": r.verify_ms},
        "kernel_timing_ms": kt,
        "trace_metadata": {"source": "gpu_solve" if r.traces else "none",
                           "note": ("per-iteration values recorded by the persistent GPU kernel" if r.traces
                                    else "no per-iteration trace was collected")},
        "iterations_trace": [{"iteration": t.iteration, "alpha": t.alpha, "beta": t.beta, "rz": t.rz, "rr": t.rr,
                              "residual": t.residual} for t in r.traces],
    }


def json_text(r: ReportInputs) -> str:
    return json.dumps(json_report(r), indent=2) + "\n"


def done_line(r: ReportInputs) -> str:
    return (f"[done] iter={r.iterations} residual_abs={_e(r.residual_l2)} residual_rel={_e(r.residual_rel)} "
            f"status={_status(r)}")


def check_line(cpu_residual_abs: float, r: ReportInputs, max_rel_diff: float, diff_tol: float) -> str:
    return (f"[check] cpu_residual_abs={_e(cpu_residual_abs)} b200_residual_abs={_e(r.residual_l2)} "
            f"max_abs_diff={_e(r.max_abs_diff)} max_rel_diff={_e(max_rel_diff)} diff_tol={_e(diff_tol)}")


def timing_line(r: ReportInputs) -> str:
    per = 1e3 * r.kernel_ms / r.iterations if r.iterations > 0 else 0.0
    return (f"[timing-ms] setup={_e(r.host_setup_ms)} solve={_e(r.total_ms)} kernel={_e(r.kernel_ms)} "
            f"iterations={r.iterations} us_per_iteration={_e(per)}")


def host_residual(dataset, x) -> float:
    """||b - A x|| in FP64 on the host (compute_residual_norm, src/CgSolverGolden.hpp:126-135)."""
    rp, ci, v = dataset.row_ptr, dataset.col_idx, dataset.values
    rows = np.repeat(np.arange(dataset.n), np.diff(rp))
    ax = np.zeros(dataset.n)
    np.add.at(ax, rows, v * x[ci])
    return float(np.linalg.norm(dataset.b - ax))


def main(argv=None) -> int:
    from . import XPLUS_TAU_ABS_RR, XPLUS_TAU_REL_TRUE, CsrDataset, PcgSolver, run_defaults
    ap = argparse.ArgumentParser(description="Solve a CSR dataset directory on the GPU and report")
    ap.add_argument("dataset")
    ap.add_argument("--tau", type=float, default=run_defaults.kTau)
    ap.add_argument("--max-iters", type=int, default=run_defaults.kMaxIters)
    ap.add_argument("--rel", action="store_true", help="tau is the FP64 true relative residual")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--text-report")
    ap.add_argument("--json-report")
    ap.add_argument("--x-ref", help="text file with a reference solution for max_abs_diff")
    ap.add_argument("--diff-tol", type=float, default=1e-6)
    a = ap.parse_args(argv)
    t0 = time.perf_counter()
    ds = CsrDataset.load(a.dataset)
    solver = PcgSolver.from_dataset(ds, device=a.device)
    t1 = time.perf_counter()
    res = solver.solve(ds.b, ds.x0, tau=a.tau, tau_mode=XPLUS_TAU_REL_TRUE if a.rel else XPLUS_TAU_ABS_RR,
                       max_iters=a.max_iters, trace=True)
    t2 = time.perf_counter()
    solver.close()
    res_abs = host_residual(ds, res.solution)
    bn = float(np.linalg.norm(ds.b))
    xref = np.loadtxt(a.x_ref) if a.x_ref else None
    diff = np.abs(res.solution - xref) if xref is not None else np.zeros(1)
    rel = diff / np.maximum(np.abs(xref), 1e-12) if xref is not None else np.zeros(1)
    t3 = time.perf_counter()
    r = ReportInputs(dataset_dir=str(a.dataset), n=ds.n, nnz=ds.nnz, effective_max_iters=res.effective_max_iters,
                     tau=a.tau, device_index=a.device, pass_=res.converged and float(diff.max()) <= a.diff_tol,
                     converged=res.converged, breakdown=res.status == "breakdown", iterations=res.iterations,
                     final_rr=res.final_rr, residual_l2=res_abs, residual_rel=res_abs / bn if bn > 0 else res_abs,
                     max_abs_diff=float(diff.max()), golden_residual_l2=math.nan if xref is None else host_residual(ds, xref),
                     total_ms=(t2 - t1) * 1e3, host_setup_ms=(t1 - t0) * 1e3, h2d_ms=0.0, kernel_ms=res.kernel_ms,
                     d2h_ms=0.0, verify_ms=(t3 - t2) * 1e3, traces=res.iteration_trace)
    print(done_line(r))
    print(check_line(r.golden_residual_l2, r, float(rel.max()), a.diff_tol))
    print(timing_line(r))
    if a.text_report:
        Path(a.text_report).parent.mkdir(parents=True, exist_ok=True)
        Path(a.text_report).write_text(text_report(r))
    if a.json_report:
        Path(a.json_report).parent.mkdir(parents=True, exist_ok=True)
        Path(a.json_report).write_text(json_text(r))
    return 0 if res.converged else 2


if __name__ == "__main__":
    sys.exit(main())
