"""FP64 CPU oracle of the learned G^T G preconditioner (test infrastructure only).

The learned preconditioner has no counterpart in the reference project: its oracle is this
plain-numpy restatement of the network, the probe loss and their gradients, written out by
hand in FP64.  It is pinned by central finite differences (tests/test_gnn_oracle.py) and is
the checker for the GPU forward / backward / Adam kernels.  Product code never imports it.

Network (hidden width H = 32, 3 message-passing layers), on the graph of an SPD matrix A in
the row order the solver is given:
  node inputs   x_i = [log a_ii - mean_k log a_kk,  (sum_j |a_ij|) / a_ii - 1]
  edge values   e_ij = a_ij / sqrt(a_ii a_jj)                               (i != j)
  input layer   h = relu(W0 x + b0)
  layer l       s_i = Wa h_i + ba + sum_{j<i} e_ij Wl h_j + sum_{j>i} e_ij Wu h_j
                h_i <- h_i + relu(s_i)
                (lower and upper neighbours get their own weights: G is lower-triangular in
                this order, so what G_ij should be depends on which neighbours precede i)
  edge head     for j < i, a_ij != 0:  z = relu(P h_i + bp + Q h_j + c e_ij + c2 f_ij),
                Ghat_ij = w . z + bw, with f_ij = sum_{m < i, m != j} e_jm e_mi (two-step paths
                from j to i through i's other lower neighbours)
  diagonal      Ghat_ii = exp(wd . h_i + bwd)
  G             G_ij = Ghat_ij / sqrt(a_jj)   (so G = Ghat D^-1/2, and Ghat = I is Jacobi)
Losses: the probe loss over K vectors v ~ N(0, I), L = sum_p ||G A G^T v_p - v_p||^2 / (K n),
and the row-normalized Kaporin loss L = (1/n) sum_i [log (G A G^T)_ii - 2 log Ghat_ii]
(kaporin_loss; the network is trained with it, and the solver scales G's rows to
(G A G^T)_ii = 1 after inference).
The forward pass uses the parameters rounded to BF16 (round to nearest even), and the node
products W h and D W take their node operand rounded to BF16 too (they run on the tensor
cores, FP32 accumulation); gradients are taken with respect to the rounded values and applied
to the FP32 master copy.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.sparse as sp

H = 32
LAYERS = 3


def layout():
    """(name, shape) of every parameter, in the order of the flat parameter vector."""
    out = [("W0", (H, 2)), ("b0", (H,))]
    for l in range(LAYERS):
        out += [(f"Wa{l}", (H, H)), (f"ba{l}", (H,)), (f"Wl{l}", (H, H)), (f"Wu{l}", (H, H))]
    out += [("P", (H, H)), ("bp", (H,)), ("Q", (H, H)), ("c", (H,)), ("c2", (H,)), ("w", (H,)), ("bw", (1,)),
            ("wd", (H,)), ("bwd", (1,))]
    return out


def n_params() -> int:
    return sum(int(np.prod(s)) for _, s in layout())


def unpack(theta):
    p, o = {}, 0
    for name, shape in layout():
        k = int(np.prod(shape))
        p[name] = np.asarray(theta[o:o + k], np.float64).reshape(shape)
        o += k
    return p


def pack(d) -> np.ndarray:
    return np.concatenate([np.asarray(d[name], np.float64).ravel() for name, _ in layout()])


def bf16_round(a) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def init_params(seed: int = 0) -> np.ndarray:
    """Seeded initial parameters (float32 values): uniform(+-1/sqrt(fan_in)) weights, zero
    biases, and a zero output layer, so the untrained network gives G = D^-1/2 (Jacobi)."""
    rng = np.random.default_rng(seed)
    d = {}
    for name, shape in layout():
        if name in ("w", "bw", "wd", "bwd") or name.startswith("b"):
            d[name] = np.zeros(shape)
        elif name in ("c", "c2"):
            d[name] = rng.uniform(-0.5, 0.5, shape)
        else:
            fan_in = shape[1]
            d[name] = rng.uniform(-1, 1, shape) / math.sqrt(fan_in)
    return pack(d).astype(np.float32)


def graph(row_ptr, col_idx, values) -> dict:
    """Graph arrays of A (CSR, any order of columns within a row)."""
    n = len(row_ptr) - 1
    A = sp.csr_matrix((np.asarray(values, np.float64), np.asarray(col_idx), np.asarray(row_ptr)), shape=(n, n))
    A.sort_indices()
    d = A.diagonal().copy()
    coo = A.tocoo()
    off = coo.row != coo.col
    r, c, v = coo.row[off], coo.col[off], coo.data[off]
    e = v / np.sqrt(d[r] * d[c])
    rowabs = np.asarray(abs(A).sum(axis=1)).ravel()
    ld = np.log(d)
    x = np.stack([ld - ld.mean(), rowabs / d - 1.0], 1)
    low = c < r
    # f_ij = (L E)_ij on the lower edges: L the strictly lower part of E = the off-diagonal
    # scaled matrix, so the sum runs over i's lower neighbours m with m != j adjacent to j
    E = sp.csr_matrix((e, (r, c)), shape=(n, n))
    L = sp.csr_matrix((e[low], (r[low], c[low])), shape=(n, n))
    lf = np.asarray((L @ E)[r[low], c[low]]).ravel()
    return dict(n=n, A=A, d=d, x=x, r=r, c=c, e=e, low=low, lr=r[low], lc=c[low], le=e[low], lf=lf)


def _agg(g, vals_lo, vals_up):
    """m_i = sum_{j<i} e_ij lo_j + sum_{j>i} e_ij up_j over the off-diagonal edges (i, j)."""
    src = np.where(g["low"][:, None], vals_lo[g["c"]], vals_up[g["c"]]) * g["e"][:, None]
    m = np.zeros((g["n"], vals_lo.shape[1]))
    np.add.at(m, g["r"], src)
    return m


def _tc(a, on):
    """An operand of the node products W h and D W, which run on the tensor cores: rounded to
    BF16 (through FP32, as the GPU holds it) when the rounded model is evaluated."""
    return bf16_round(a) if on else a


def forward(theta, g, round_bf16=True):
    """round_bf16: the parameters, and the node activations entering the products W h, rounded
    to BF16 as on the GPU; False: the exact FP64 model (for finite differences)."""
    p = unpack(bf16_round(theta) if round_bf16 else np.asarray(theta, np.float64))
    cache = {"p": p, "rb": round_bf16}
    pre0 = g["x"] @ p["W0"].T + p["b0"]
    h = np.maximum(pre0, 0.0)
    cache["pre0"], hs, ss = pre0, [h], []
    for l in range(LAYERS):
        hb = _tc(h, round_bf16)
        s = hb @ p[f"Wa{l}"].T + p[f"ba{l}"] + _agg(g, hb @ p[f"Wl{l}"].T, hb @ p[f"Wu{l}"].T)
        h = h + np.maximum(s, 0.0)
        ss.append(s)
        hs.append(h)
    cache["hs"], cache["ss"] = hs, ss
    hb = _tc(h, round_bf16)
    ph = hb @ p["P"].T + p["bp"]
    qh = hb @ p["Q"].T
    zpre = ph[g["lr"]] + qh[g["lc"]] + np.outer(g["le"], p["c"]) + np.outer(g["lf"], p["c2"])
    z = np.maximum(zpre, 0.0)
    go = z @ p["w"] + p["bw"][0]
    gd = np.exp(h @ p["wd"] + p["bwd"][0])
    cache.update(zpre=zpre, z=z, gd=gd)
    return go, gd, cache


def g_matrix(g, go, gd):
    n = g["n"]
    isq = 1.0 / np.sqrt(g["d"])
    rows = np.concatenate([g["lr"], np.arange(n)])
    cols = np.concatenate([g["lc"], np.arange(n)])
    vals = np.concatenate([go, gd]) * isq[cols]
    return sp.csr_matrix((vals, (rows, cols)), shape=(n, n))


def _splitmix64(x):
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = x
    z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(0xFFFFFFFFFFFFFFFF)
    return z ^ (z >> np.uint64(31))


def probes(n: int, k: int, seed: int) -> np.ndarray:
    """[n, k] standard normal probes, the generator the GPU uses: element (i, p) with index
    q = i*k + p takes u1, u2 from splitmix64 of (seed, 2q) and (seed, 2q+1), mapped to
    (0, 1] with 53 bits, then Box-Muller  sqrt(-2 ln u1) cos(2 pi u2)."""
    with np.errstate(over="ignore"):
        q = np.arange(n * k, dtype=np.uint64)
        s = np.uint64(seed) * np.uint64(0xD1B54A32D192ED03) & np.uint64(0xFFFFFFFFFFFFFFFF)
        a = _splitmix64(s ^ (np.uint64(2) * q))
        b = _splitmix64(s ^ (np.uint64(2) * q + np.uint64(1)))
    u1 = ((a >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    u2 = ((b >> np.uint64(11)).astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    return (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)).reshape(n, k)


def loss(theta, g, v, round_bf16=True) -> float:
    go, gd, _ = forward(theta, g, round_bf16)
    G = g_matrix(g, go, gd)
    r = G @ (g["A"] @ (G.T @ v)) - v
    return float((r * r).sum() / (v.shape[1] * g["n"]))


def loss_and_grad(theta, g, v, round_bf16=True):
    """Probe loss and its gradient with respect to the (rounded) parameters, FP64, by hand."""
    n, K = g["n"], v.shape[1]
    go, gd, cache = forward(theta, g, round_bf16)
    G = g_matrix(g, go, gd)
    A = g["A"]
    w1 = G.T @ v
    w2 = A @ w1
    r = G @ w2 - v
    L = float((r * r).sum() / (K * n))
    y = A @ (G.T @ r)
    scale = 2.0 / (K * n)
    isq = 1.0 / np.sqrt(g["d"])
    # dL/dG_ij = scale * sum_p (r_ip w2_jp + v_ip y_jp) on the pattern (i, j <= i)
    dG_off = scale * ((r[g["lr"]] * w2[g["lc"]]).sum(1) + (v[g["lr"]] * y[g["lc"]]).sum(1))
    dG_dia = scale * ((r * w2).sum(1) + (v * y).sum(1))
    dgo = dG_off * isq[g["lc"]]
    dexp = dG_dia * isq * gd
    return L, _backward(g, cache, dgo, dexp)


def scaled_matrix(g):
    """A^ = D^-1/2 A D^-1/2 (unit diagonal) as CSR."""
    isq = 1.0 / np.sqrt(g["d"])
    return (sp.diags(isq) @ g["A"] @ sp.diags(isq)).tocsr()


def ghat_matrix(g, go, gd):
    """Ghat (the head's output before the D^-1/2 column scaling) as CSR."""
    n = g["n"]
    rows = np.concatenate([g["lr"], np.arange(n)])
    cols = np.concatenate([g["lc"], np.arange(n)])
    return sp.csr_matrix((np.concatenate([go, gd]), (rows, cols)), shape=(n, n))


def kaporin_terms(g, go, gd):
    """Per-row B_i = (G A G^T)_ii = ghat_i^T A^ ghat_i and U = Ghat A^ restricted to Ghat's
    pattern: U_ij = (A^ ghat_i)_j for j in the pattern of row i (lower edges, then diagonal)."""
    Gh = ghat_matrix(g, go, gd)
    U = (Gh @ scaled_matrix(g)).tocsr()
    B = np.asarray(U.multiply(Gh).sum(axis=1)).ravel()
    u_off = np.asarray(U[g["lr"], g["lc"]]).ravel()
    u_dia = U.diagonal()
    return B, u_off, u_dia


def kaporin_loss(theta, g, round_bf16=True) -> float:
    """Row-normalized Kaporin loss L = (1/n) sum_i [log (G A G^T)_ii - 2 log G^_ii].
    Per row it is the log of (g A g) / g_ii^2 over the row's pattern, which is invariant to the
    row's scale and is smallest for the exact FSAI row (the factorized sparse approximate
    inverse minimizes Kaporin's condition number det-ratio of G A G^T over the pattern).  Summed
    over rows it is, up to a constant, n log K(G A G^T) once the rows are scaled to unit
    (G A G^T)_ii, which the solver does after inference."""
    go, gd, _ = forward(theta, g, round_bf16)
    B, _, _ = kaporin_terms(g, go, gd)
    return float((np.log(B) - 2.0 * np.log(gd)).mean())


def kaporin_loss_and_grad(theta, g, round_bf16=True):
    """Kaporin loss and its gradient, FP64, by hand:
      dL/dGhat_ij = 2 U_ij / (n B_i)  (j < i),   dL/dt_i = 2 U_ii gd_i / (n B_i) - 2 / n
    with t_i the diagonal head's pre-exponential value (Ghat_ii = gd_i = exp t_i)."""
    n = g["n"]
    go, gd, cache = forward(theta, g, round_bf16)
    B, u_off, u_dia = kaporin_terms(g, go, gd)
    L = float((np.log(B) - 2.0 * np.log(gd)).mean())
    dgo = 2.0 * u_off / (n * B[g["lr"]])
    dexp = 2.0 * u_dia * gd / (n * B) - 2.0 / n
    return L, _backward(g, cache, dgo, dexp)


def refine_rows(g, go, gd, sweeps=1):
    """Gauss-Seidel sweeps on each row's quadratic form ghat^T A^[P_i, P_i] ghat at fixed
    Ghat_ii: for the lower entries j of row i in ascending order, ghat_ij -= (A^ ghat_i)_j
    (A^_jj = 1).  Returns the new lower values (graph order); the diagonal is unchanged."""
    n = g["n"]
    lr, lc = g["lr"], g["lc"]
    cnt = np.bincount(lr, minlength=n)
    lptr = np.concatenate([[0], np.cumsum(cnt)])
    Ah = scaled_matrix(g)
    go = np.array(go, np.float64)
    for _ in range(sweeps):
        for k in range(int(cnt.max()) if n else 0):
            rows = np.nonzero(cnt > k)[0]
            e_k = lptr[rows] + k                    # the entry being set, row by row
            j = lc[e_k]
            u = gd[rows] * np.asarray(Ah[j, rows]).ravel()   # the diagonal entry of the pattern
            for q in range(int(cnt.max())):
                has = cnt[rows] > q
                eq = lptr[rows[has]] + q
                u[has] += go[eq] * np.asarray(Ah[j[has], lc[eq]]).ravel()
            go[e_k] -= u
    return go


def normalize_rows(g, go, gd):
    """Rows of Ghat scaled to (G A G^T)_ii = 1 (what the solver applies after inference)."""
    B, _, _ = kaporin_terms(g, go, gd)
    s = 1.0 / np.sqrt(B)
    return go * s[g["lr"]], gd * s


def _backward(g, cache, dgo, dexp):
    """Parameter gradient from dL/dGhat on the lower edges (dgo) and dL/dt on the diagonal
    (dexp = dL/dGhat_ii * Ghat_ii): the same chain for every loss."""
    n = g["n"]
    p = cache["p"]
    grads = {name: np.zeros(shape) for name, shape in layout()}
    h = cache["hs"][-1]
    z, zpre = cache["z"], cache["zpre"]
    # edge head
    grads["w"] = z.T @ dgo
    grads["bw"] = np.array([dgo.sum()])
    dz = np.outer(dgo, p["w"]) * (zpre > 0)
    grads["c"] = dz.T @ g["le"]
    grads["c2"] = dz.T @ g["lf"]
    dph = np.zeros((n, H))
    np.add.at(dph, g["lr"], dz)
    dqh = np.zeros((n, H))
    np.add.at(dqh, g["lc"], dz)
    grads["P"] = dph.T @ h
    grads["bp"] = dph.sum(0)
    grads["Q"] = dqh.T @ h
    grads["wd"] = h.T @ dexp
    grads["bwd"] = np.array([dexp.sum()])
    rb = cache["rb"]
    dh = _tc(dph, rb) @ p["P"] + _tc(dqh, rb) @ p["Q"] + np.outer(dexp, p["wd"])
    # layers, last to first
    for l in reversed(range(LAYERS)):
        hin = cache["hs"][l]
        s = cache["ss"][l]
        ds = dh * (s > 0)
        # m_i = sum_{j<i} e_ij (Wl h)_j + sum_{j>i} e_ij (Wu h)_j
        # -> d(Wl h)_j = sum_{i>j} e_ij ds_i ; d(Wu h)_j = sum_{i<j} e_ij ds_i
        up_of_j = g["r"] > g["c"]          # edge (r=i, c=j) with i > j contributes to dhl_j
        src = ds[g["r"]] * g["e"][:, None]
        dhl = np.zeros((n, H))
        dhu = np.zeros((n, H))
        np.add.at(dhl, g["c"][up_of_j], src[up_of_j])
        np.add.at(dhu, g["c"][~up_of_j], src[~up_of_j])
        grads[f"Wa{l}"] = ds.T @ hin
        grads[f"ba{l}"] = ds.sum(0)
        grads[f"Wl{l}"] = dhl.T @ hin
        grads[f"Wu{l}"] = dhu.T @ hin
        dh = dh + _tc(ds, rb) @ p[f"Wa{l}"] + _tc(dhl, rb) @ p[f"Wl{l}"] + _tc(dhu, rb) @ p[f"Wu{l}"]
    dpre0 = dh * (cache["pre0"] > 0)
    grads["W0"] = dpre0.T @ g["x"]
    grads["b0"] = dpre0.sum(0)
    return pack(grads)


def adam(theta, m, v, grad, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step (step counts from 1) in FP64; returns the new (theta, m, v)."""
    m = b1 * m + (1 - b1) * grad
    v = b2 * v + (1 - b2) * grad * grad
    mh = m / (1 - b1 ** step)
    vh = v / (1 - b2 ** step)
    return theta - lr * mh / (np.sqrt(vh) + eps), m, v


def fsai_lower(row_ptr, col_idx, values):
    """Exact factorized sparse approximate inverse on A's lower pattern (Kolotilina-Yeremin):
    row i of G solves A[P_i, P_i] g = e_i over P_i = {j <= i : a_ij != 0}, scaled so that
    (G A G^T)_ii = 1.  Returns the values in A's CSR order of the entries with j <= i."""
    n = len(row_ptr) - 1
    A = sp.csr_matrix((values, col_idx, row_ptr), shape=(n, n))
    out = []
    for i in range(n):
        cols = np.asarray(col_idx[row_ptr[i]:row_ptr[i + 1]])
        pat = cols[cols <= i]
        sub = A[pat][:, pat].toarray()
        rhs = (pat == i).astype(np.float64)
        y = np.linalg.solve(sub, rhs)
        y /= math.sqrt(y[pat == i][0])
        out.append(y)
    return np.concatenate(out) if out else np.zeros(0)
