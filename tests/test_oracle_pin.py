"""Pins the oracle: the C restatement against the reference's own code (built from its
sources into oracle/_ref) and against the committed golden fixtures that code produced."""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = sorted((Path(__file__).parent / "golden").glob("golden_*.npz"))


class DS:
    def __init__(self, z):
        self.row_ptr, self.col_idx, self.values = z["row_ptr"], z["col_idx"], z["values"]
        self.b, self.x0 = z["b"], z["x0"]
        self.n = len(self.row_ptr) - 1


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_golden_restatement_is_bit_exact(oracle, path):
    z = np.load(path)
    r = oracle.golden(DS(z), float(z["tau"]), int(z["max_iters"]))
    assert r["iterations"] == int(z["golden_iterations"])
    assert np.array_equal(r["x"], z["golden_x"])
    assert np.array_equal(r["trace"], z["golden_trace"])


@pytest.mark.parametrize("path", [p for p in GOLDEN if "mk_x" in np.load(p)], ids=lambda p: p.stem)
def test_multi_kernel_restatement(oracle, path):
    z = np.load(path)
    r = oracle.multi_kernel(DS(z), float(z["tau"]), int(z["max_iters"]))
    assert r["iterations"] == int(z["mk_iterations"])
    assert r["status"] == int(z["mk_status"])
    assert np.array_equal(r["x"], z["mk_x"])
    # the reference's trace passes through its %.12e log line
    np.testing.assert_allclose(r["trace"], z["mk_trace"], rtol=1e-11, atol=0)


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_cuper_style_spmv_bit_exact(oracle, path):
    z = np.load(path)
    y = oracle.cuper_spmv(DS(z), z["x_true"])
    assert np.array_equal(y, z["cuper_spmv_y"])


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_control_flow_restatement(oracle, path):
    """The control kernel accumulates its FP32 SpMV in packed-stream order; the restatement
    accumulates in CSR order.  Same control flow and status; iterates agree to FP32 level."""
    z = np.load(path)
    r = oracle.control(DS(z), float(z["tau"]), int(z["max_iters"]), spmv_mode=1)
    assert r["status"] == int(z["ctl_status"])
    assert abs(r["iterations"] - int(z["ctl_iterations"])) <= max(2, int(z["ctl_iterations"]) // 20)
    xr = z["ctl_x"]
    assert np.linalg.norm(r["x"] - xr) <= 1e-4 * np.linalg.norm(xr)


@pytest.mark.ref
def test_reference_build_matches_restatement_live(oracle, sys0):
    d, _ = sys0
    a = oracle.golden(d, 1e-10)
    b = oracle.golden(d, 1e-10, use_ref=True)
    assert a["iterations"] == b["iterations"] and np.array_equal(a["x"], b["x"])
    m1 = oracle.multi_kernel(d, 1e-10)
    m2 = oracle.multi_kernel(d, 1e-10, use_ref=True)
    assert np.array_equal(m1["x"], m2["x"]) and m1["status"] == m2["status"]


@pytest.mark.ref
def test_reference_multi_kernel_rejects_large_n(oracle):
    from project_xplus_b200 import generators as g
    d, _ = g.fem2d(33)
    with pytest.raises(RuntimeError, match="kMaxN"):
        oracle.multi_kernel(d, 1e-10, use_ref=True)
    # the restatement (and the GPU path) have no such cap
    r = oracle.multi_kernel(d, 1e-10)
    assert r["status"] == 0


def test_golden_edge_cases(oracle, sys0):
    d, _ = sys0
    with pytest.raises(RuntimeError, match="tau"):
        oracle.golden(d, 0.0)
    # converged before the first iteration: b = A x0
    r = oracle.golden(d, 1e-10, b=np.zeros(d.n))
    assert r["iterations"] == 0 and r["converged"]
    # max_iters = 0 means max(4n, 1000)
    r = oracle.golden(d, 1e-300, 0)
    assert r["iterations"] == 4 * d.n or r["final_rr"] <= 1e-300
