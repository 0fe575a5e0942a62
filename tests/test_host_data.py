"""Host-side data path: loader, binary cache, Jacobi diagonal, generators, RCM, SELL-C-sigma,
Cuper packed-format import.  No GPU needed."""
from pathlib import Path

import numpy as np
import pytest

import project_xplus_b200 as xp
from project_xplus_b200 import generators as g
from oracle import sell_rcm_oracle as SO

GOLDEN = sorted((Path(__file__).parent / "golden").glob("golden_*.npz"))


def test_text_loader_roundtrip(tmp_path, sys0):
    d, _ = sys0
    d.save_text(tmp_path)
    e = xp.CsrDataset.load(tmp_path)
    assert e.n == d.n and e.nnz == d.nnz
    for k in ("row_ptr", "col_idx", "values", "b", "x0"):
        assert np.array_equal(getattr(e, k), getattr(d, k))


@pytest.mark.ref
def test_text_loader_matches_reference_loader(tmp_path, sys0, oracle):
    import ctypes as C
    d, _ = sys0
    d.save_text(tmp_path)
    lib = oracle.reflib()
    n, nnz = C.c_int(), C.c_int()
    assert lib.ref_load(str(tmp_path).encode(), C.byref(n), C.byref(nnz), None, None, None, None, None) == 0
    rp = np.empty(n.value + 1, np.int32); ci = np.empty(nnz.value, np.int32)
    v = np.empty(nnz.value); b = np.empty(n.value); x0 = np.empty(n.value)
    P = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    assert lib.ref_load(str(tmp_path).encode(), C.byref(n), C.byref(nnz), P(rp), P(ci), P(v), P(b), P(x0)) == 0
    e = xp.CsrDataset.load(tmp_path)
    for a, bb in ((e.row_ptr, rp), (e.col_idx, ci), (e.values, v), (e.b, b), (e.x0, x0)):
        assert np.array_equal(a, bb)


@pytest.mark.parametrize("mutate,msg", [
    (lambda f: f["row_ptr.txt"].__setitem__(0, "1"), "row_ptr\\[0\\] must be 0"),
    (lambda f: f["row_ptr.txt"].__setitem__(-1, "5"), "row_ptr\\[n\\] must equal nnz"),
    (lambda f: f["col_idx.txt"].__setitem__(0, "99999"), "col_idx out of range"),
    (lambda f: f["values.txt"].pop(), "size mismatch"),
    (lambda f: f["b.txt"].pop(), "b.txt length must equal n"),
    (lambda f: f["x0.txt"].pop(), "x0.txt length must equal n"),
    (lambda f: f.__setitem__("b.txt", []), "empty array file"),
    (lambda f: f.pop("values.txt"), "failed to open"),
])
def test_loader_errors_match_reference_messages(tmp_path, mutate, msg):
    d, _ = g.fem2d(4)
    files = {"row_ptr.txt": [str(v) for v in d.row_ptr.tolist()],
             "col_idx.txt": [str(v) for v in d.col_idx.tolist()],
             "values.txt": [repr(v) for v in d.values.tolist()], "b.txt": [repr(v) for v in d.b.tolist()],
             "x0.txt": [repr(v) for v in d.x0.tolist()]}
    mutate(files)
    for k, vals in files.items():
        (tmp_path / k).write_text(" ".join(vals) + "\n")
    with pytest.raises(xp.XplusError, match=msg):
        xp.CsrDataset.load(tmp_path)


def test_binary_cache_roundtrip(tmp_path, sys0):
    d, _ = sys0
    d.save_binary(tmp_path / "a.xcsr")
    e = xp.CsrDataset.load_binary(tmp_path / "a.xcsr")
    for k in ("row_ptr", "col_idx", "values", "b", "x0"):
        assert np.array_equal(getattr(e, k), getattr(d, k))
    (tmp_path / "bad").write_bytes(b"nope")
    with pytest.raises(xp.XplusError, match="not an xplus binary"):
        xp.CsrDataset.load_binary(tmp_path / "bad")


def test_jacobi_diag_and_errors(sys0):
    d, _ = sys0
    diag = d.extract_jacobi_diag()
    for i in (0, 17, d.n - 1):
        k = [k for k in range(d.row_ptr[i], d.row_ptr[i + 1]) if d.col_idx[k] == i][0]
        assert diag[i] == d.values[k]
    e = xp.CsrDataset(d.row_ptr, d.col_idx, d.values.copy(), d.b, d.x0)
    k = [k for k in range(e.row_ptr[5], e.row_ptr[6]) if e.col_idx[k] == 5][0]
    e.values[k] = 0.0
    with pytest.raises(xp.XplusError, match="zero diagonal entry at row 5"):
        e.extract_jacobi_diag()
    ci = d.col_idx.copy()
    ci[k] = 4
    f = xp.CsrDataset(d.row_ptr, ci, d.values, d.b, d.x0)
    with pytest.raises(xp.XplusError, match="missing diagonal entry at row 5"):
        f.extract_jacobi_diag()


@pytest.mark.parametrize("dim,gsz", [(2, 32), (2, 9), (3, 6)])
def test_fem_generators_are_spd(dim, gsz):
    d, xt = (g.fem2d(gsz) if dim == 2 else g.fem3d(gsz))
    import scipy.sparse as sp
    A = sp.csr_matrix((d.values, d.col_idx, d.row_ptr)).toarray()
    assert d.n == gsz ** dim
    assert np.allclose(A, A.T, rtol=0, atol=0)
    assert np.linalg.eigvalsh(A).min() > 0
    np.testing.assert_allclose(A @ xt, d.b, rtol=0, atol=1e-12 * np.abs(d.b).max())
    assert (xt >= -1).all() and (xt <= 1).all()
    # columns sorted in every row
    for i in range(d.n):
        row = d.col_idx[d.row_ptr[i]:d.row_ptr[i + 1]]
        assert (np.diff(row) > 0).all()
    nz = d.nnz / d.n
    assert (6.0 <= nz <= 7.5) if dim == 2 else (11 <= nz <= 15.5)


def test_fem3d_interior_rows_have_15_entries():
    d, _ = g.fem3d(7)
    lens = np.diff(d.row_ptr).reshape(7, 7, 7)
    assert (lens[1:-1, 1:-1, 1:-1] == 15).all()


def test_generator_is_deterministic():
    a, xa = g.fem2d(20, sigma=2.0, seed=3, perm_seed=1, rcm=True)
    b, xb = g.fem2d(20, sigma=2.0, seed=3, perm_seed=1, rcm=True)
    assert np.array_equal(a.values, b.values) and np.array_equal(a.col_idx, b.col_idx)
    assert np.array_equal(xa, xb)
    c, _ = g.fem2d(20, sigma=2.0, seed=4)
    assert not np.array_equal(a.values, c.values)


@pytest.mark.parametrize("gsz,perm_seed", [(30, 1), (17, 5), (3, 0)])
def test_rcm_bit_exact_against_restatement(gsz, perm_seed):
    d, _ = g.fem2d(gsz, perm_seed=perm_seed)
    assert np.array_equal(g.rcm(d.row_ptr, d.col_idx), SO.rcm(d.row_ptr, d.col_idx))


def test_rcm_disconnected_components():
    # two disjoint 2D systems side by side (block diagonal)
    a, _ = g.fem2d(5)
    n = a.n
    rp = np.concatenate([a.row_ptr, a.row_ptr[1:] + a.nnz])
    ci = np.concatenate([a.col_idx, a.col_idx + n])
    assert np.array_equal(g.rcm(rp, ci), SO.rcm(rp, ci))


def test_rcm_reduces_bandwidth():
    d, _ = g.fem2d(40, perm_seed=1)
    def bw(rp, ci):
        return max(abs(int(ci[k]) - i) for i in range(len(rp) - 1) for k in range(rp[i], rp[i + 1]))
    p = g.rcm(d.row_ptr, d.col_idx)
    rp, ci, _ = g.permute_symmetric(d.row_ptr, d.col_idx, d.values, p)
    assert bw(rp, ci) < 3 * 40 < bw(d.row_ptr, d.col_idx)


def test_permute_symmetric_bit_exact():
    d, _ = g.fem2d(12, perm_seed=2)
    p = np.random.default_rng(0).permutation(d.n).astype(np.int32)
    a = g.permute_symmetric(d.row_ptr, d.col_idx, d.values, p)
    b = SO.permute_symmetric(d.row_ptr, d.col_idx, d.values, p)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.parametrize("chunk", [1, 2, 4])
@pytest.mark.parametrize("diag_split", [False, True])
@pytest.mark.parametrize("sigma", [1, 32, 256])
def test_sell_bit_exact_against_restatement(chunk, diag_split, sigma):
    d, _ = g.fem2d(23, sigma=1.5, perm_seed=4)
    a = g.sell_build(d.row_ptr, d.col_idx, d.values, sigma=sigma, chunk=chunk, diag_split=diag_split)
    b = SO.sell_build(d.row_ptr, d.col_idx, d.values, sigma=sigma, chunk=chunk, diag_split=diag_split)
    for k in ("perm", "slice_ptr", "slice_width", "col", "val"):
        assert np.array_equal(a[k], b[k]), k
    if diag_split:
        assert np.array_equal(a["diag"], b["diag"])


def test_sell_ragged_rows_and_empty_row():
    # rows of length 0..5 incl. an empty row; n not a multiple of 32
    rng = np.random.default_rng(1)
    n = 45
    rows = [sorted(rng.choice(n, size=rng.integers(0, 6), replace=False).tolist()) for _ in range(n)]
    rows[7] = []
    rp = np.cumsum([0] + [len(r) for r in rows]).astype(np.int32)
    ci = np.array([c for r in rows for c in r], np.int32)
    v = rng.standard_normal(len(ci))
    for chunk in (1, 2, 4):
        a = g.sell_build(rp, ci, v, sigma=16, chunk=chunk)
        b = SO.sell_build(rp, ci, v, sigma=16, chunk=chunk)
        for k in ("perm", "slice_ptr", "col", "val"):
            assert np.array_equal(a[k], b[k])
        # every CSR entry appears once (multiset of (new_row, new_col, val))
        inv = np.empty(n, np.int64); inv[a["perm"]] = np.arange(n)
        assert int((a["val"] != 0).sum()) == int((v != 0).sum())


@pytest.mark.parametrize("path", GOLDEN, ids=[p.stem for p in GOLDEN])
def test_cuper_unpack_roundtrips_reference_packer(path):
    """Decoding the reference packer's words gives back the CSR entries (multiset, FP32)."""
    z = np.load(path)
    n = len(z["row_ptr"]) - 1
    rows, cols, vals = g.cuper_unpack(n, int(z["pack_batch_count"]), z["pack_ptr"], z["pack_words"],
                                      int(z["pack_channel_words"]))
    rp, ci, v = z["row_ptr"], z["col_idx"], z["values"]
    want = sorted((i, int(ci[k]), float(np.float32(v[k]))) for i in range(n) for k in range(rp[i], rp[i + 1]))
    got = sorted(zip(rows.tolist(), cols.tolist(), [float(x) for x in vals]))
    assert got == want


def test_cuper_row_map_matches_restatement():
    import random
    random.seed(0)
    for _ in range(1000):
        row = random.randrange(0, 1 << 20)
        pid = row // 2
        ch = (pid % 8) * 2 + (pid // 8) % 2
        lane = (pid // 16) % 8
        prow = (row // 256) * 2 + (row & 1)
        assert SO.cuper_global_row(ch, lane, prow) == row
