"""The learned preconditioner M^-1 = G^T G: network parameters, the GPU trainer, and the
solver-side entry points (xplus_gnn_*, xplus_pcg_set_gnn / set_gtg, xplus_fsai_lower).

G is lower-triangular on A's lower pattern in the solver's row order, so G^T G is SPD by
construction and is applied as two sliced SpMVs.  A 3-layer message-passing network (hidden
width 32) predicts G's values; it is trained on the GPU (hand-written forward, backward and
Adam kernels) on systems from the project's generators, with the row-normalized Kaporin loss
(1/n) sum_i [log (G A G^T)_ii - 2 log Ghat_ii] (or the probe loss ||G A G^T v - v||^2 over
v ~ N(0, I)); the solver scales the predicted rows to (G A G^T)_ii = 1.  Plain Jacobi-PCG
takes over inside the solve when the learned solve stagnates or passes its iteration cap, and
the FP64 true residual decides convergence either way.
"""
from __future__ import annotations

import ctypes as C
import json
import math
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import check, lib, ptr

H = 32
LAYERS = 3
WEIGHTS_DIR = Path(__file__).resolve().parent / "weights"
DEFAULT_WEIGHTS = WEIGHTS_DIR / "gtg_gnn.npz"


def layout():
    """(name, shape) of every parameter block in the flat vector (the order gnn.cu uses)."""
    out = [("W0", (H, 2)), ("b0", (H,))]
    for l in range(LAYERS):
        out += [(f"Wa{l}", (H, H)), (f"ba{l}", (H,)), (f"Wl{l}", (H, H)), (f"Wu{l}", (H, H))]
    out += [("P", (H, H)), ("bp", (H,)), ("Q", (H, H)), ("c", (H,)), ("c2", (H,)), ("w", (H,)), ("bw", (1,)),
            ("wd", (H,)), ("bwd", (1,))]
    return out


def param_count() -> int:
    return int(lib.xplus_gnn_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """Seeded float32 parameters: weights uniform in +-1/sqrt(fan_in), biases zero, edge
    weights c and c2 uniform in +-0.5, and a zero output layer (w, bw, wd, bwd), so the untrained
    network predicts G = D^-1/2: exactly Jacobi."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in layout():
        if name in ("w", "bw", "wd", "bwd") or name.startswith("b"):
            a = np.zeros(shape)
        elif name in ("c", "c2"):
            a = rng.uniform(-0.5, 0.5, shape)
        else:
            a = rng.uniform(-1, 1, shape) / math.sqrt(shape[1])
        parts.append(np.asarray(a, np.float64).ravel())
    theta = np.concatenate(parts).astype(np.float32)
    assert theta.size == param_count()
    return theta


def save_weights(path, params, meta: dict) -> None:
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez(path, params=np.asarray(params, np.float32), meta=json.dumps(meta))


def load_weights(path=DEFAULT_WEIGHTS):
    z = np.load(path)
    params = np.asarray(z["params"], np.float32)
    if params.size != param_count():
        raise ValueError(f"{path}: {params.size} parameters, the network has {param_count()}")
    return params, json.loads(str(z["meta"]))


def fsai_lower(row_ptr, col_idx, values) -> np.ndarray:
    """Exact FSAI on A's lower pattern (host), in g_low order."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    n = len(rp) - 1
    out = np.empty(int(np.count_nonzero(ci <= np.repeat(np.arange(n), np.diff(rp)))), np.float64)
    check(lib.xplus_fsai_lower(n, ptr(rp), ptr(ci), ptr(v), ptr(out)))
    return out


def jacobi_g(row_ptr, col_idx, values) -> np.ndarray:
    """G = D^-1/2 in g_low order (G^T G is the Jacobi inverse)."""
    rp = np.asarray(row_ptr)
    ci = np.asarray(col_idx)
    n = len(rp) - 1
    rows = np.repeat(np.arange(n), np.diff(rp))
    keep = ci <= rows
    vals = np.asarray(values, np.float64)[keep]
    isdiag = ci[keep] == rows[keep]
    return np.where(isdiag, 1.0 / np.sqrt(np.where(isdiag, vals, 1.0)), 0.0)


class GnnTrainer:
    """Training systems resident on one GPU plus the network state (xplus_gnn_trainer)."""

    LOSSES = {"probe": _lib.XPLUS_GNN_LOSS_PROBE, "kaporin": _lib.XPLUS_GNN_LOSS_KAPORIN}

    @staticmethod
    def _csr_arrays(systems):
        systems = [(np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32),
                    np.ascontiguousarray(v, np.float64)) for rp, ci, v in systems]
        k = len(systems)
        ns = np.array([len(s[0]) - 1 for s in systems], np.int32)
        rps = (C.c_void_p * k)(*[ptr(s[0]) for s in systems])
        cis = (C.c_void_p * k)(*[ptr(s[1]) for s in systems])
        vs = (C.c_void_p * k)(*[ptr(s[2]) for s in systems])
        return systems, k, ns, rps, cis, vs

    def __init__(self, systems, *, probes=8, device=0, params=None, loss="probe"):
        self.systems, k, ns, rps, cis, vs = self._csr_arrays(systems)
        h = C.c_void_p()
        check(lib.xplus_gnn_trainer_create(k, rps, cis, vs, ptr(ns), int(probes), int(device), C.byref(h)))
        self._h = h
        self.probes = probes
        self.set_params(init_params(0) if params is None else params)
        self.set_loss(loss)

    def set_loss(self, loss: str) -> None:
        """"probe": ||G A G^T v - v||^2 over random probes; "kaporin": the row-normalized
        Kaporin loss (1/n) sum_i [log (G A G^T)_ii - 2 log Ghat_ii]."""
        check(lib.xplus_gnn_set_loss(self._h, self.LOSSES[loss]))
        self.loss = loss

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            lib.xplus_gnn_trainer_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(params, np.float32)
        if p.size != param_count():
            raise ValueError("wrong parameter count")
        check(lib.xplus_gnn_set_params(self._h, ptr(p)))

    def params(self) -> np.ndarray:
        p = np.empty(param_count(), np.float32)
        check(lib.xplus_gnn_get_params(self._h, ptr(p)))
        return p

    def loss_grad(self, sys: int, seed: int, grad=True):
        loss = C.c_double()
        g = np.empty(param_count(), np.float32) if grad else None
        check(lib.xplus_gnn_loss_grad(self._h, int(sys), int(seed), C.byref(loss), ptr(g)))
        return loss.value, g

    def adam(self, grad, lr: float) -> None:
        g = np.ascontiguousarray(grad, np.float32)
        check(lib.xplus_gnn_adam(self._h, ptr(g), float(lr)))

    def load(self, systems) -> None:
        """Replaces the resident training systems; parameters and Adam state are kept."""
        self.systems, k, ns, rps, cis, vs = self._csr_arrays(systems)
        check(lib.xplus_gnn_trainer_load(self._h, k, rps, cis, vs, ptr(ns)))

    def train(self, steps: int, lr=3e-3, lr_final=1e-4, seed=1, first_step=0, total_steps=None) -> np.ndarray:
        """Adam steps [first_step, first_step + steps) of a cosine schedule over total_steps
        (default: this call's steps alone)."""
        losses = np.empty(steps, np.float64)
        total = steps if total_steps is None else int(total_steps)
        check(lib.xplus_gnn_train_window(self._h, int(steps), float(lr), float(lr_final), int(seed),
                                         int(first_step), total, ptr(losses)))
        return losses

    def predict(self, sys: int) -> np.ndarray:
        """G of system `sys` as the network outputs it, rows not normalized (the solver's
        set_gnn scales them to (G A G^T)_ii = 1)."""
        n = C.c_int64()
        check(lib.xplus_gnn_predict(self._h, int(sys), None, C.byref(n)))
        g = np.empty(n.value, np.float64)
        check(lib.xplus_gnn_predict(self._h, int(sys), ptr(g), C.byref(n)))
        return g
