"""The FP64 oracle of the learned preconditioner, pinned without a GPU: its hand-written
backward against central finite differences, its probe generator, its parameter layout and
initial values against the product's, and the host FSAI against the oracle's restatement."""
import numpy as np
import pytest

from oracle import gnn_oracle as O


@pytest.fixture(scope="module")
def small():
    from project_xplus_b200 import generators as gen
    d, _ = gen.fem2d(6, sigma=1.5, seed=3, perm_seed=2, rcm=True)
    return d, O.graph(d.row_ptr, d.col_idx, d.values)


def test_backward_matches_finite_differences(small):
    d, g = small
    rng = np.random.default_rng(0)
    theta = O.init_params(1).astype(np.float64) + rng.normal(0, 0.05, O.n_params())
    v = O.probes(g["n"], 3, 7)
    _, grad = O.loss_and_grad(theta, g, v, round_bf16=False)
    idx = np.concatenate([rng.choice(O.n_params(), 80, replace=False), np.arange(O.n_params() - 130, O.n_params())])
    h = 1e-6
    for k in idx:
        e = np.zeros_like(theta)
        e[k] = h
        fd = (O.loss(theta + e, g, v, False) - O.loss(theta - e, g, v, False)) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-6 + 1e-4 * abs(fd), (k, fd, grad[k])


def test_kaporin_backward_matches_finite_differences(small):
    d, g = small
    rng = np.random.default_rng(1)
    theta = O.init_params(2).astype(np.float64) + rng.normal(0, 0.05, O.n_params())
    _, grad = O.kaporin_loss_and_grad(theta, g, round_bf16=False)
    idx = np.concatenate([rng.choice(O.n_params(), 80, replace=False), np.arange(O.n_params() - 130, O.n_params())])
    h = 1e-6
    for k in idx:
        e = np.zeros_like(theta)
        e[k] = h
        fd = (O.kaporin_loss(theta + e, g, False) - O.kaporin_loss(theta - e, g, False)) / (2 * h)
        assert abs(fd - grad[k]) <= 1e-7 + 1e-5 * abs(fd), (k, fd, grad[k])


def test_kaporin_loss_is_smallest_at_fsai_and_row_scale_free():
    """Per row the loss is log (g A g / g_ii^2) on the row's pattern: invariant to the row's
    scale, and its minimum over the pattern is the exact FSAI row (so FSAI is the floor the
    network is trained toward); the untrained network (Jacobi) is above it."""
    from project_xplus_b200 import generators as gen
    d, _ = gen.fem2d(10, sigma=2.0, seed=5, perm_seed=3, rcm=True)
    g = O.graph(d.row_ptr, d.col_idx, d.values)
    n = d.n
    rows = np.repeat(np.arange(n), np.diff(d.row_ptr))
    keep = d.col_idx <= rows
    fs = O.fsai_lower(d.row_ptr, d.col_idx, d.values)
    r_, c_ = rows[keep], d.col_idx[keep]
    # FSAI in Ghat form (Ghat = G D^1/2), split into lower edges (graph order) and diagonal
    sq = np.sqrt(g["d"])
    fmap = {(int(a), int(b)): v * sq[b] for a, b, v in zip(r_, c_, fs)}
    go_f = np.array([fmap[(int(a), int(b))] for a, b in zip(g["lr"], g["lc"])])
    gd_f = np.array([fmap[(i, i)] for i in range(n)])
    B, _, _ = O.kaporin_terms(g, go_f, gd_f)
    l_fsai = float((np.log(B) - 2 * np.log(gd_f)).mean())
    np.testing.assert_allclose(B, 1.0, rtol=1e-10)  # FSAI rows are already unit-normalized
    B2, _, _ = O.kaporin_terms(g, 3.0 * go_f, 3.0 * gd_f)
    assert abs(float((np.log(B2) - 2 * np.log(3.0 * gd_f)).mean()) - l_fsai) < 1e-12
    rng = np.random.default_rng(0)
    for _ in range(5):
        go_p = go_f * (1 + 0.05 * rng.standard_normal(go_f.size))
        Bp, _, _ = O.kaporin_terms(g, go_p, gd_f)
        assert float((np.log(Bp) - 2 * np.log(gd_f)).mean()) > l_fsai
    assert O.kaporin_loss(O.init_params(0), g) > l_fsai
    # normalize_rows gives unit (G A G^T)_ii
    gn, dn = O.normalize_rows(g, go_p, gd_f)
    np.testing.assert_allclose(O.kaporin_terms(g, gn, dn)[0], 1.0, rtol=1e-12)


def test_refine_rows_lowers_every_row_and_reaches_fsai():
    """Each Gauss-Seidel sweep lowers every row's Kaporin term (or keeps it), and repeated
    sweeps converge to the exact FSAI row (the minimizer on the pattern)."""
    from project_xplus_b200 import generators as gen
    d, _ = gen.fem2d(9, sigma=2.0, seed=6, perm_seed=2, rcm=True)
    g = O.graph(d.row_ptr, d.col_idx, d.values)
    rng = np.random.default_rng(2)
    theta = O.init_params(3).astype(np.float64) + rng.normal(0, 0.1, O.n_params())
    go, gd, _ = O.forward(theta, g, round_bf16=False)

    def ell(a, b):
        B, _, _ = O.kaporin_terms(g, a, b)
        return np.log(B) - 2 * np.log(b)
    prev = ell(go, gd)
    cur = go
    for _ in range(3):
        cur = O.refine_rows(g, cur, gd, 1)
        now = ell(cur, gd)
        assert np.all(now <= prev + 1e-12)
        prev = now
    many = O.refine_rows(g, go, gd, 400)
    fs = O.fsai_lower(d.row_ptr, d.col_idx, d.values)
    n = d.n
    rows = np.repeat(np.arange(n), np.diff(d.row_ptr))
    keep = d.col_idx <= rows
    sq = np.sqrt(g["d"])
    fmap = {(int(a), int(b)): v * sq[b] for a, b, v in zip(rows[keep], d.col_idx[keep], fs)}
    gd_f = np.array([fmap[(i, i)] for i in range(n)])
    go_f = np.array([fmap[(int(a), int(b))] for a, b in zip(g["lr"], g["lc"])])
    # same row directions: ratios to the diagonal agree
    np.testing.assert_allclose(many / gd[g["lr"]], go_f / gd_f[g["lr"]], rtol=1e-6, atol=1e-9)


def test_untrained_network_is_jacobi(small):
    d, g = small
    go, gd, _ = O.forward(O.init_params(0), g)
    assert np.all(go == 0.0) and np.all(gd == 1.0)
    G = O.g_matrix(g, go, gd)
    np.testing.assert_allclose(G.diagonal(), 1.0 / np.sqrt(g["d"]))


def test_layout_and_init_match_the_product():
    from project_xplus_b200 import learned as L
    assert L.param_count() == O.n_params()
    assert L.layout() == O.layout()
    np.testing.assert_array_equal(L.init_params(5), O.init_params(5))


def test_probes_are_standard_normal_and_seeded():
    v = O.probes(4000, 8, 11)
    assert v.shape == (4000, 8)
    assert abs(v.mean()) < 0.03 and abs(v.std() - 1) < 0.03
    np.testing.assert_array_equal(v, O.probes(4000, 8, 11))
    assert not np.array_equal(v, O.probes(4000, 8, 12))


def test_bf16_rounding():
    # bf16 spacing at 1 is 2^-7: 1 + 2^-8 and 1 + 3 * 2^-8 are ties, rounded to the even neighbour
    x = np.array([1.0, 1.00390625, 1.01171875, 1.001953125, -3.14159, 1e-3], np.float32)
    r = O.bf16_round(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.015625 and r[3] == 1.0
    assert np.all(np.abs(r - x) <= np.abs(x) * 2.0 ** -8)


def test_host_fsai_matches_oracle():
    from project_xplus_b200 import generators as gen
    from project_xplus_b200 import learned as L
    for d in (gen.fem2d(12, sigma=2.0, seed=4, perm_seed=1, rcm=True)[0], gen.fem3d(5, sigma=1.5, seed=2)[0]):
        a = L.fsai_lower(d.row_ptr, d.col_idx, d.values)
        b = O.fsai_lower(d.row_ptr, d.col_idx, d.values)
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-14)
        # (G A G^T)_ii = 1
        g = O.graph(d.row_ptr, d.col_idx, d.values)
        n = d.n
        rows = np.repeat(np.arange(n), np.diff(d.row_ptr))
        keep = d.col_idx <= rows
        import scipy.sparse as sp
        G = sp.csr_matrix((a, (rows[keep], d.col_idx[keep])), shape=(n, n))
        np.testing.assert_allclose((G @ g["A"] @ G.T).diagonal(), 1.0, rtol=1e-10)


def test_jacobi_g_is_d_inverse_sqrt():
    from project_xplus_b200 import generators as gen
    from project_xplus_b200 import learned as L
    d, _ = gen.fem2d(7)
    gl = L.jacobi_g(d.row_ptr, d.col_idx, d.values)
    n = d.n
    rows = np.repeat(np.arange(n), np.diff(d.row_ptr))
    keep = d.col_idx <= rows
    diag = d.col_idx[keep] == rows[keep]
    g = O.graph(d.row_ptr, d.col_idx, d.values)
    np.testing.assert_allclose(gl[diag], 1 / np.sqrt(g["d"]))
    assert np.all(gl[~diag] == 0)
