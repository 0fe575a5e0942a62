"""Batched solver (xplus_batch_*): every system of a batch solved in one persistent launch
reaches the FP64 true-residual tolerance, agrees with the single-system solver and with the
FP64 oracle solve, and the graph-captured device path and the autotuner give the same answers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _systems(specs):
    from project_xplus_b200 import generators as g
    out = []
    for side, sigma, seed in specs:
        d, xt = g.fem2d(side, sigma=sigma, jitter=0.3, seed=seed, x_seed=seed)
        out.append((d, xt))
    return out


SPECS = [(12, 1.0, 1), (45, 2.0, 2), (20, 0.5, 3), (64, 2.5, 4), (33, 1.5, 5), (7, 1.0, 6), (96, 1.2, 7)]


@pytest.fixture(scope="module")
def batch_systems():
    return _systems(SPECS)


def _make(batch_systems, **kw):
    from project_xplus_b200.batch import BatchSolver
    return BatchSolver([(d.row_ptr, d.col_idx, d.values) for d, _ in batch_systems], **kw)


def _b(batch_systems):
    return np.concatenate([d.b for d, _ in batch_systems])


@pytest.mark.parametrize("vt", ["f32", "f16", "bf16"])
def test_every_system_converges(gpu, batch_systems, vt):
    s = _make(batch_systems, values_dtype=vt)
    r = s.solve(_b(batch_systems), tau=1e-8)
    assert list(r["status"]) == [0] * len(SPECS), r["status_names"]
    assert np.all(r["true_rel"] <= 1e-8)
    for (d, xt), x in zip(batch_systems, s.split(r["x"])):
        # the solution itself: the same residual check on the host, in FP64
        res = np.linalg.norm(d.b - _spmv(d, x)) / np.linalg.norm(d.b)
        assert res <= 1.5e-8
    assert r["kernel_ms"] > 0 and np.all(r["system_ms"] > 0)


def _spmv(d, x):
    y = np.zeros(d.n)
    rows = np.repeat(np.arange(d.n), np.diff(d.row_ptr))
    np.add.at(y, rows, d.values * x[d.col_idx])
    return y


def test_matches_single_system_solver(gpu, batch_systems):
    """Same iteration, same FP32/FP64 split: iteration counts agree with the single-system
    persistent kernel up to the order of the dot-product sums, and both solutions are within
    the tolerance's reach of the FP64 oracle solution."""
    from scipy.sparse import csr_matrix
    from scipy.sparse.linalg import spsolve

    from project_xplus_b200 import PcgSolver, XPLUS_TAU_REL_TRUE
    s = _make(batch_systems)
    r = s.solve(_b(batch_systems), tau=1e-8)
    for k, ((d, xt), x) in enumerate(zip(batch_systems, s.split(r["x"]))):
        single = PcgSolver(d.row_ptr, d.col_idx, d.values, resident=False)
        rs = single.solve(d.b, tau=1e-8, tau_mode=XPLUS_TAU_REL_TRUE)
        single.close()
        assert rs.converged
        it_b, it_s = int(r["iterations"][k]), rs.iterations
        assert abs(it_b - it_s) <= max(3, 0.05 * it_s), (k, it_b, it_s)
        A = csr_matrix((d.values, d.col_idx, d.row_ptr), shape=(d.n, d.n))
        x64 = spsolve(A.tocsc(), d.b)
        scale = np.linalg.norm(x64)
        err_b = np.linalg.norm(x - x64) / scale
        err_s = np.linalg.norm(rs.solution - x64) / scale
        assert err_b <= 10 * max(err_s, 1e-9), (k, err_b, err_s)


def test_x0_and_absolute_tolerance(gpu, batch_systems):
    from project_xplus_b200 import XPLUS_TAU_ABS_RR
    s = _make(batch_systems)
    b = _b(batch_systems)
    rng = np.random.default_rng(0)
    x0 = rng.uniform(-1, 1, s.total_n)
    r = s.solve(b, x0, tau=1e-12, tau_mode=XPLUS_TAU_ABS_RR)
    assert list(r["status"]) == [0] * len(SPECS)
    # x0 = the exact solution converges at once
    xs = np.concatenate([xt for _, xt in batch_systems])
    r2 = s.solve(b, xs, tau=1e-12, tau_mode=XPLUS_TAU_ABS_RR)
    assert list(r2["iterations"]) == [0] * len(SPECS)
    # max_iters caps every system: status 1 (max_iter)
    r3 = s.solve(b, tau=1e-30, tau_mode=XPLUS_TAU_ABS_RR, max_iters=5)
    assert list(r3["status"]) == [1] * len(SPECS) and list(r3["iterations"]) == [5] * len(SPECS)


def test_device_graph_path(gpu, batch_systems):
    import torch
    s = _make(batch_systems)
    b = _b(batch_systems)
    host = s.solve(b, tau=1e-8)
    st = torch.cuda.Stream()
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros_like(d_b)
    for rep in range(3):  # first call captures the graph, the next ones replay it
        d_x.zero_()
        torch.cuda.synchronize()
        s.solve_device(d_b, d_x, tau=1e-8, stream=st)
        st.synchronize()
        r = s.results()
        assert list(r["status"]) == [0] * len(SPECS)
        np.testing.assert_array_equal(d_x.cpu().numpy(), host["x"])  # deterministic


def test_device_graph_path_rejects_host_pointers(gpu, batch_systems):
    """xplus_batch_solve_device: host arrays are an argument error, before any capture."""
    import torch
    from project_xplus_b200 import XplusError
    from project_xplus_b200._lib import XPLUS_ERR_ARG
    s = _make(batch_systems)
    b = _b(batch_systems)
    with pytest.raises(XplusError) as e:
        s.solve_device(b, np.zeros_like(b), tau=1e-8)
    assert e.value.code == XPLUS_ERR_ARG and "host memory" in str(e.value)
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros_like(d_b)
    s.solve_device(d_b, d_x, tau=1e-8)
    torch.cuda.synchronize()
    assert list(s.results()["status"]) == [0] * len(SPECS)


@pytest.mark.parametrize("count,cluster,tpb", [(1, 16, 512), (2, 8, 512), (7, 16, 256)])
def test_lane_of_the_largest_systems(gpu, batch_systems, count, cluster, tpb):
    """The largest systems in a concurrent launch of their own with bigger clusters (16 CTAs is
    beyond the portable limit): every system still reaches the tolerance, the split systems'
    iteration counts stay within the dot-product rounding of the one-launch solve, and the
    graph-captured device path agrees with the host path bit for bit."""
    import torch
    s = _make(batch_systems)
    b = _b(batch_systems)
    one = s.solve(b, tau=1e-8)
    s.set_split_lane(count, cluster, tpb)
    lane = s.split_lane()
    assert lane["count"] == count and lane["cluster"] == cluster and lane["grid"] % cluster == 0
    two = s.solve(b, tau=1e-8)
    assert list(two["status"]) == [0] * len(SPECS)
    assert np.all(two["true_rel"] <= 1e-8)
    for k in range(len(SPECS)):
        assert abs(int(two["iterations"][k]) - int(one["iterations"][k])) <= max(3, 0.03 * one["iterations"][k])
    for (d, _), x in zip(batch_systems, s.split(two["x"])):
        assert np.linalg.norm(d.b - _spmv(d, x)) / np.linalg.norm(d.b) <= 1.5e-8
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros_like(d_b)
    st = torch.cuda.Stream()
    for _ in range(2):
        d_x.zero_()
        torch.cuda.synchronize()
        s.solve_device(d_b, d_x, tau=1e-8, stream=st)
        st.synchronize()
        np.testing.assert_array_equal(d_x.cpu().numpy(), two["x"])
    s.set_split_lane(0)
    assert s.split_lane()["count"] == 0
    s.close()


@pytest.mark.parametrize("vt", ["f32", "f16", "bf16"])
@pytest.mark.parametrize("cluster,tpb,split", [(1, 512, 0), (2, 256, 0), (4, 256, 2), (8, 512, 0)])
def test_resident_kernel(gpu, batch_systems, vt, cluster, tpb, split):
    """The cluster-resident kernel (vectors and the search direction's window in shared
    memory, one cluster barrier per iteration): every system reaches the tolerance, its
    iteration count stays within the dot-product rounding of the global-memory kernel's, the
    two solutions are equally close to the direct solve (two solutions at residual 1e-8 may
    differ by up to cond(A) x 1e-8), repeated solves are bit-identical, staging the bands'
    matrices in shared memory changes no bit, and the graph-captured device path gives the host
    path's x bit for bit."""
    import torch
    from scipy.sparse import csr_matrix
    from scipy.sparse.linalg import spsolve
    s = _make(batch_systems, values_dtype=vt)
    b = _b(batch_systems)
    s.set_launch(cluster, tpb)
    if split:
        s.set_split_lane(split, 16, 256)
    ref = s.solve(b, tau=1e-8)
    s.set_resident(True)
    info = s.resident()
    assert info["on"] and 0 < info["smem"] <= 232448 and (info["smem_split"] > 0) == bool(split)
    r = s.solve(b, tau=1e-8)
    assert list(r["status"]) == [0] * len(SPECS), r["status_names"]
    assert np.all(r["true_rel"] <= 1e-8)
    for k, ((d, _), x, x_ref) in enumerate(zip(batch_systems, s.split(r["x"]), s.split(ref["x"]))):
        it, it_ref = int(r["iterations"][k]), int(ref["iterations"][k])
        assert abs(it - it_ref) <= max(4, 0.06 * it_ref), (k, it, it_ref)
        assert np.linalg.norm(d.b - _spmv(d, x)) / np.linalg.norm(d.b) <= 1.5e-8
        x64 = spsolve(csr_matrix((d.values, d.col_idx, d.row_ptr), shape=(d.n, d.n)).tocsc(), d.b)
        err, err_ref = (np.linalg.norm(v - x64) / np.linalg.norm(x64) for v in (x, x_ref))
        assert err <= 10 * max(err_ref, 1e-7), (k, err, err_ref)
    again = s.solve(b, tau=1e-8)
    np.testing.assert_array_equal(again["x"], r["x"])
    # each band's matrix staged in shared memory (the default) or read from global memory:
    # the same products in the same order, so the same x bit for bit
    staged = s.staged()
    assert staged["on"] and staged["all"] + staged["some"] > 0, staged
    s.set_stage_matrix(False)
    assert s.resident()["smem"] <= info["smem"]
    unstaged = s.solve(b, tau=1e-8)
    assert s.staged() == dict(on=False, all=0, some=0)
    np.testing.assert_array_equal(unstaged["x"], r["x"])
    np.testing.assert_array_equal(unstaged["iterations"], r["iterations"])
    s.set_stage_matrix(True)
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros_like(d_b)
    st = torch.cuda.Stream()
    for _ in range(2):
        d_x.zero_()
        torch.cuda.synchronize()
        s.solve_device(d_b, d_x, tau=1e-8, stream=st)
        st.synchronize()
        np.testing.assert_array_equal(d_x.cpu().numpy(), r["x"])
    s.set_resident(False)
    assert not s.resident()["on"]
    np.testing.assert_array_equal(s.solve(b, tau=1e-8)["x"], ref["x"])
    s.close()


def test_resident_kernel_refuses_systems_that_do_not_fit(gpu):
    """A 128x128 system's band does not fit one CTA's shared memory at cluster size 1: the
    resident kernel is refused with XPLUS_ERR_ARG before any launch and the handle keeps its
    kernel; at clusters of 4 it fits and solves."""
    from project_xplus_b200 import XplusError
    from project_xplus_b200.batch import BatchSolver
    sys2 = _systems([(128, 1.0, 8), (20, 1.0, 9)])
    s = BatchSolver([(d.row_ptr, d.col_idx, d.values) for d, _ in sys2])
    s.set_launch(1, 512)
    with pytest.raises(XplusError) as e:
        s.set_resident(True)
    assert e.value.code == 10 and "does not fit" in str(e.value)
    assert not s.resident()["on"]
    s.set_launch(4, 256)
    s.set_resident(True)
    r = s.solve(np.concatenate([d.b for d, _ in sys2]), tau=1e-8)
    assert list(r["status"]) == [0, 0] and np.all(r["true_rel"] <= 1e-8)
    with pytest.raises(XplusError):
        s.set_launch(1, 512)  # refused: the 128x128 band no longer fits
    assert s.info()["cluster"] == 4 and s.resident()["on"]
    s.close()


def test_launch_shapes_and_autotune(gpu, batch_systems):
    from project_xplus_b200 import XplusError
    from project_xplus_b200.batch import autotune_build
    s = _make(batch_systems)
    b = _b(batch_systems)
    xs = []
    for cl, tpb in ((1, 512), (2, 256), (8, 128)):
        s.set_launch(cl, tpb)
        info = s.info()
        assert info["cluster"] == cl and info["block_threads"] == tpb and info["grid"] % cl == 0
        r = s.solve(b, tau=1e-8)
        assert list(r["status"]) == [0] * len(SPECS)
        xs.append(r["x"])
    with pytest.raises(XplusError):
        s.set_launch(3, 512)
    t = s.autotune(iters=20)
    assert t["cluster"] in (1, 2, 4, 8) and t["block_threads"] in (128, 256, 512) and t["ms"] > 0
    t = s.autotune(tau=1e-8)
    assert t["ms"] > 0 and s.info()["cluster"] == t["cluster"]
    assert s.solve(b, tau=1e-8)["status"].tolist() == [0] * len(SPECS)
    best, info = autotune_build([(d.row_ptr, d.col_idx, d.values) for d, _ in batch_systems], b,
                                sigmas=(1, 256), chunks=(2, 4), iters=10)
    assert len(info["table"]) == 4
    assert best.solve(b, tau=1e-8)["status"].tolist() == [0] * len(SPECS)
    best.close()


@pytest.mark.parametrize("vt", ["f32", "bf16"])
def test_many_uneven_systems(gpu, vt):
    """More systems than clusters, sides log-uniform in [45, 128]: the queue hands out every
    system exactly once and each converges, with FP32 values and with BF16 values (two-term
    entries in cancelling rows, flexible re-conjugation at replacements)."""
    from project_xplus_b200 import generators as g
    from project_xplus_b200.batch import BatchSolver
    sides, sigmas = g.batch_sides(96, 45, 128, seed=11)
    systems = [g.fem2d(int(sd), sigma=float(sg), seed=100 + k, x_seed=100 + k)[0]
               for k, (sd, sg) in enumerate(zip(sides, sigmas))]
    s = BatchSolver([(d.row_ptr, d.col_idx, d.values) for d in systems], values_dtype=vt)
    r = s.solve(np.concatenate([d.b for d in systems]), tau=1e-8)
    assert np.all(r["status"] == 0) and np.all(r["true_rel"] <= 1e-8)
    assert np.all(r["iterations"] > 0)
