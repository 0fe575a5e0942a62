"""GPU parity of the persistent Jacobi-PCG kernel and the SELL SpMV against the oracle.

Tolerances (relative unless stated):
  * FP64 values + FP64 vectors vs the golden (src/CgSolverGolden.hpp): same iteration count
    (+-1), per-iteration residual within 1e-9 for the first 50 iterations, x within 1e-8.
  * FP32 values + FP64 vectors (the control kernel's arithmetic) vs the golden on FP32-rounded
    values: per-iteration residual within 1e-9 for 50 iterations.
  * FP32 values + FP32 vectors (the plain product) vs the golden on FP32-rounded values:
    per-iteration residual within 1e-5 for the first 40 iterations on the n=1024 system
    (FP32 storage alone drifts past 1e-5 near iteration 45 there: the oracle at FP32
    precision shows it), x from a TAU_REL_TRUE solve within 1e-6 of the FP64 oracle solve.
"""
from pathlib import Path

import numpy as np
import pytest

import project_xplus_b200 as xp
from project_xplus_b200 import generators as g

pytestmark = pytest.mark.gpu

GOLDEN = sorted((Path(__file__).parent / "golden").glob("golden_*.npz"))


def ds_of(z):
    return xp.CsrDataset(z["row_ptr"], z["col_idx"], z["values"], z["b"], z["x0"])


def f32_rounded(d):
    return xp.CsrDataset(d.row_ptr, d.col_idx, d.values.astype(np.float32).astype(np.float64), d.b, d.x0)


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
@pytest.mark.parametrize("chunk", [1, 4])
def test_fp64_solve_matches_golden(gpu, path, chunk):
    z = np.load(path)
    d = ds_of(z)
    s = xp.PcgSolver.from_dataset(d, values_dtype="f64", vector_dtype="f64", chunk=chunk)
    r = s.solve(d.b, d.x0, tau=float(z["tau"]), max_iters=int(z["max_iters"]), trace=True)
    gi = int(z["golden_iterations"])
    assert abs(r.iterations - gi) <= 1
    k = min(50, gi, r.iterations)
    got = np.array([t.residual for t in r.iteration_trace[:k]])
    np.testing.assert_allclose(got, z["golden_trace"][:k, 4], rtol=1e-9)
    gx = z["golden_x"]
    assert np.linalg.norm(r.solution - gx) <= 1e-8 * np.linalg.norm(gx) + 1e-300
    want_status = "converged" if int(z["max_iters"]) == 0 else "max_iter"
    assert r.status == want_status


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_fp32_values_fp64_vectors_match_golden_on_rounded_values(gpu, oracle, path):
    z = np.load(path)
    d = ds_of(z)
    d32 = f32_rounded(d)
    gr = oracle.golden(d32, float(z["tau"]), int(z["max_iters"]))
    s = xp.PcgSolver.from_dataset(d, values_dtype="f32", vector_dtype="f64", keep_fp64=True)
    r = s.solve(d.b, d.x0, tau=float(z["tau"]), max_iters=int(z["max_iters"]), trace=True)
    k = min(50, gr["iterations"], r.iterations)
    got = np.array([t.residual for t in r.iteration_trace[:k]])
    np.testing.assert_allclose(got, gr["trace"][:k, 4], rtol=1e-9)
    assert abs(r.iterations - gr["iterations"]) <= 2


def test_plain_fp32_residual_history_matches_golden(gpu, oracle, sys0):
    d, _ = sys0
    d32 = f32_rounded(d)
    gr = oracle.golden(d32, 1e-30, 60)
    s = xp.PcgSolver.from_dataset(d, values_dtype="f32", vector_dtype="f32")
    r = s.solve(d.b, None, tau=1e-30, max_iters=60, trace=True)
    assert r.iterations == 60 and r.status == "max_iter"
    got = np.array([t.residual for t in r.iteration_trace[:40]])
    np.testing.assert_allclose(got, gr["trace"][:40, 4], rtol=1e-5)
    # alpha, beta, rz follow the same recurrences
    for j, name in ((0, "alpha"), (1, "beta"), (2, "rz")):
        v = np.array([getattr(t, name) for t in r.iteration_trace[:40]])
        np.testing.assert_allclose(v, gr["trace"][:40, j], rtol=1e-4, err_msg=name)


def test_plain_fp32_final_x_matches_fp64_oracle(gpu, oracle, sys0):
    d, xt = sys0
    ref = oracle.golden(d, 1e-30, 2000)  # FP64 oracle solve run to its floor
    s = xp.PcgSolver.from_dataset(d, values_dtype="f32", vector_dtype="f32", keep_fp64=True)
    r = s.solve(d.b, None, tau=1e-12, tau_mode=xp.XPLUS_TAU_REL_TRUE, max_iters=5000)
    assert r.status == "converged"
    assert r.residual_rel <= 1e-12
    assert np.linalg.norm(r.solution - ref["x"]) <= 1e-6 * np.linalg.norm(ref["x"])
    # the kernel's FP64 exit residual agrees with the oracle's
    res = oracle.residual_norm(d, r.solution) / np.linalg.norm(d.b)
    assert res <= 1e-12 and abs(res - r.residual_rel) <= 1e-3 * res + 1e-18


@pytest.mark.parametrize("vdt,xdt,tol", [("f64", "f64", 1e-14), ("f32", "f64", 1e-14), ("f32", "f32", 2e-6),
                                         ("bf16", "f32", 2e-6)])
@pytest.mark.parametrize("chunk", [1, 2, 4])
def test_sell_spmv_matches_oracle(gpu, oracle, vdt, xdt, tol, chunk):
    d, xt = g.fem2d(45, sigma=2.0, perm_seed=1, rcm=True)
    s = xp.PcgSolver.from_dataset(d, values_dtype=vdt, vector_dtype=xdt, chunk=chunk)
    y = s.spmv(xt)
    vals = d.values
    if vdt == "f32":
        vals = vals.astype(np.float32).astype(np.float64)
    if vdt == "bf16":
        # off-diagonals rounded to bf16, diagonal kept (row-sum compensated: A~ 1 = A 1)
        import torch
        t = torch.tensor(vals).to(torch.bfloat16).double().numpy()
        rows = np.repeat(np.arange(d.n), np.diff(d.row_ptr))
        off = d.col_idx != rows
        v2 = vals.copy()
        v2[off] = t[off]
        corr = np.zeros(d.n)
        np.add.at(corr, rows[off], vals[off] - t[off])
        dg = ~off
        v2[dg] = vals[dg] + corr[rows[dg]]
        vals = v2
    xin = xt.astype(np.float32).astype(np.float64) if xdt == "f32" else xt
    want = oracle.spmv(xp.CsrDataset(d.row_ptr, d.col_idx, vals, d.b, d.x0), xin)
    scale = np.abs(vals).max() * np.abs(xin).max() * 8
    assert np.abs(y - want).max() <= tol * scale


def test_true_residual_mode_reaches_tolerance(gpu, oracle):
    d, xt = g.fem2d(150, sigma=2.0, perm_seed=1, rcm=True)
    for vdt in ("f32", "bf16"):
        s = xp.PcgSolver.from_dataset(d, values_dtype=vdt, vector_dtype="f32", replace_every=50, replace_drop=1e-4)
        r = s.solve(d.b, None, tau=1e-8, tau_mode=xp.XPLUS_TAU_REL_TRUE, max_iters=20000)
        assert r.status == "converged", (vdt, r.status, r.residual_rel)
        res = oracle.residual_norm(d, r.solution) / np.linalg.norm(d.b)
        assert res <= 1e-8, (vdt, res)
        assert r.replacements >= 1


def test_fp32_recurrence_vs_true_residual_gap(gpu, oracle):
    """In the reference's absolute-rr mode the FP32 recurrence can claim convergence while
    the FP64 true residual lags behind; the kernel reports both."""
    d, xt = g.fem2d(150, sigma=2.0, perm_seed=1, rcm=True)
    s = xp.PcgSolver.from_dataset(d, values_dtype="f32", vector_dtype="f32")
    tau_abs = (1e-8 * np.linalg.norm(d.b)) ** 2
    r = s.solve(d.b, None, tau=tau_abs, max_iters=20000)
    assert r.status == "converged" and r.final_rr <= tau_abs
    res = oracle.residual_norm(d, r.solution) / np.linalg.norm(d.b)
    assert abs(res - r.residual_rel) <= 1e-2 * res


def test_status_codes(gpu, sys0):
    d, _ = sys0
    s = xp.PcgSolver.from_dataset(d)
    r = s.solve(d.b, None, tau=1e-30, max_iters=7)
    assert r.status == "max_iter" and r.iterations == 7
    r = s.solve(np.zeros(d.n), None, tau=1e-10)
    assert r.status == "converged" and r.iterations == 0
    b = d.b.copy()
    b[3] = np.nan
    r = s.solve(b, None, tau=1e-10, max_iters=10)
    assert r.status == "breakdown"
    with pytest.raises(xp.XplusError):
        s.solve(d.b, None, tau=0.0)
    # max_iters <= 0 means max(4n, 1000) (src/CgSolverGolden.hpp:47)
    r = s.solve(d.b, None, tau=1e-10, max_iters=0)
    assert r.effective_max_iters == max(4 * d.n, 1000) and r.status == "converged"


def test_nonzero_x0_and_repeat_solves_are_deterministic(gpu):
    d, xt = g.fem2d(64, sigma=1.0)
    s = xp.PcgSolver.from_dataset(d, values_dtype="f32", vector_dtype="f32")
    x0 = np.cos(np.arange(d.n) * 0.1)
    r1 = s.solve(d.b, x0, tau=1e-12, max_iters=500, trace=True)
    r2 = s.solve(d.b, x0, tau=1e-12, max_iters=500, trace=True)
    assert r1.iterations == r2.iterations
    assert np.array_equal(r1.solution, r2.solution)
    assert [t.rr for t in r1.iteration_trace] == [t.rr for t in r2.iteration_trace]


def test_cfg_scale_solve_property(gpu, oracle):
    """The 1108x1108 system (n = 1,227,664): FP32 plain kernel with FP64 residual replacement
    reaches 1e-8 FP64 true relative residual; checked on the host in FP64."""
    d, xt = g.system_2d_large()
    s = xp.PcgSolver.from_dataset(d, values_dtype="f32", vector_dtype="f32", chunk=1)
    r = s.solve(d.b, None, tau=1e-8, tau_mode=xp.XPLUS_TAU_REL_TRUE, max_iters=20000)
    assert r.status == "converged", (r.status, r.residual_rel, r.iterations)
    res = oracle.residual_norm(d, r.solution) / np.linalg.norm(d.b)
    assert res <= 1e-8


def test_timeout_path_reports_status(gpu, sys0):
    """A grid barrier that never completes (one block skips its arrival; test-only switch)
    ends the launch with XPLUS_TIMEOUT after the bounded wait, and the context stays usable."""
    import ctypes as C
    from project_xplus_b200 import _lib
    d, _ = sys0
    s = xp.PcgSolver.from_dataset(d, barrier_timeout_s=0.2)
    assert _lib.lib.xplus_pcg_debug_skip_arrival(s.handle, 0) == 0
    r = s.solve(d.b, None, tau=1e-10, max_iters=50)
    assert r.status == "timeout"
    assert _lib.lib.xplus_pcg_debug_skip_arrival(s.handle, -1) == 0
    r = s.solve(d.b, None, tau=1e-10)
    assert r.status == "converged"
