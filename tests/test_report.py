"""Reports in the reference's formats (text sections and JSON keys of its report writer,
archived/host/report_io.hpp:83-282; [done]/[check]/[timing-ms] console lines), filled from
a solve result.  The GPU test runs the command-line solve on a dataset directory."""
import json
import math

import pytest

from project_xplus_b200 import report as R
from project_xplus_b200.solver import IterationTrace


def _inputs(**kw):
    base = dict(dataset_dir="data/x", n=1024, nnz=6976, effective_max_iters=4096, tau=1e-10, device_index=0,
                pass_=True, converged=True, breakdown=False, iterations=52, final_rr=3.2e-11, residual_l2=5.6e-6,
                residual_rel=1.2e-7, max_abs_diff=1e-9, golden_residual_l2=5.5e-6, total_ms=1.5, host_setup_ms=10.25,
                h2d_ms=0.0, kernel_ms=0.75, d2h_ms=0.0, verify_ms=0.5,
                traces=[IterationTrace(0, 0.5, 0.25, 1.0, 2.0, math.sqrt(2.0))])
    base.update(kw)
    return R.ReportInputs(**base)


def test_text_report_layout():
    t = R.text_report(_inputs())
    sections = [l for l in t.splitlines() if l.startswith("[")]
    assert sections == ["[Problem]", "[Accuracy]", "[Host Timing ms]", "[Kernel Timing ms]"]
    keys = [l.split(":")[0].strip() for l in t.splitlines() if ":" in l]
    assert keys[:6] == ["dataset", "n / nnz", "max_iters", "tau", "device_index", "pass"]
    assert "tau                : 1.000000000000e-10" in t
    assert "status             : converged" in t
    assert "host_setup         : 10.250" in t
    for name in ("spmv", "init", "dot", "update_xrz", "update_p"):
        assert f"{name}_total" in t and f"{name}_avg" in t


def test_json_report_keys():
    d = json.loads(R.json_text(_inputs()))
    assert list(d) == ["dataset", "result", "host_timing_ms", "kernel_timing_ms", "trace_metadata", "iterations_trace"]
    assert list(d["dataset"]) == ["path", "xclbin", "n", "nnz", "max_iters", "tau", "device_index"]
    assert list(d["result"]) == ["pass", "converged", "status", "iterations", "final_rr", "final_residual_norm",
                                 "residual_rel", "solution_max_abs_diff", "golden_residual_norm"]
    assert list(d["host_timing_ms"]) == ["total", "host_setup", "buffer_h2d", "kernel_total", "buffer_d2h", "verify"]
    kt = d["kernel_timing_ms"]
    assert kt["timing_model"] == "single_control_kernel" and kt["split_timing_available"] is False
    assert d["iterations_trace"][0] == {"iteration": 0, "alpha": 0.5, "beta": 0.25, "rz": 1.0, "rr": 2.0,
                                        "residual": math.sqrt(2.0)}


def test_console_lines():
    r = _inputs(converged=False, breakdown=True)
    assert R.done_line(r) == ("[done] iter=52 residual_abs=5.600000000000e-06 residual_rel=1.200000000000e-07 "
                              "status=breakdown")
    assert R.check_line(5.5e-6, r, 2e-9, 1e-6).startswith("[check] cpu_residual_abs=5.500000000000e-06 b200_residual_abs=")
    assert R.timing_line(r).startswith("[timing-ms] setup=1.025000000000e+01")


@pytest.mark.gpu
def test_command_line_solve_writes_reports(gpu, tmp_path, sys0):
    d, xt = sys0
    d.save_text(tmp_path / "ds")
    import numpy as np
    np.savetxt(tmp_path / "xref.txt", xt)
    rc = R.main([str(tmp_path / "ds"), "--rel", "--tau", "1e-11", "--max-iters", "5000", "--text-report",
                 str(tmp_path / "r.txt"), "--json-report", str(tmp_path / "r.json"), "--x-ref", str(tmp_path / "xref.txt")])
    assert rc == 0
    j = json.loads((tmp_path / "r.json").read_text())
    assert j["result"]["converged"] and j["result"]["iterations"] > 0
    assert j["result"]["solution_max_abs_diff"] < 1e-6
    assert len(j["iterations_trace"]) == j["result"]["iterations"]
    assert "[Accuracy]" in (tmp_path / "r.txt").read_text()
