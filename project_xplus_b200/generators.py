"""Synthetic SPD systems and the host-side data path (SELL-C-sigma, RCM, Cuper import).

All of it runs natively in libxplus_b200.so; these are thin array-in/array-out wrappers.
The named workloads below are the systems the solver is measured on.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, lib, ptr
from .solver import CsrDataset


def _gen(fn, g, sigma, jitter, seed, perm_seed, rcm, x_seed):
    n, nnz = C.c_int(), C.c_int()
    args = (int(g), float(sigma), float(jitter), int(seed), int(perm_seed), int(bool(rcm)), int(x_seed))
    check(fn(*args, C.byref(n), C.byref(nnz), None, None, None, None, None))
    rp = np.empty(n.value + 1, np.int32)
    ci = np.empty(nnz.value, np.int32)
    v = np.empty(nnz.value, np.float64)
    b = np.empty(n.value, np.float64)
    xt = np.empty(n.value, np.float64)
    check(fn(*args, C.byref(n), C.byref(nnz), ptr(rp), ptr(ci), ptr(v), ptr(b), ptr(xt)))
    return CsrDataset(rp, ci, v, b, np.zeros(n.value)), xt


def fem2d(g, sigma=1.0, jitter=0.3, seed=0, perm_seed=-1, rcm=False, x_seed=0):
    """P1 triangles on a jittered (g+2)^2 grid, Dirichlet ring eliminated: n = g^2."""
    return _gen(lib.xplus_gen_fem2d, g, sigma, jitter, seed, perm_seed, rcm, x_seed)


def fem3d(g, sigma=1.5, jitter=0.25, seed=0, perm_seed=-1, rcm=False, x_seed=0):
    """P1 Kuhn tetrahedra on a jittered (g+2)^3 grid, Dirichlet boundary eliminated: n = g^3."""
    return _gen(lib.xplus_gen_fem3d, g, sigma, jitter, seed, perm_seed, rcm, x_seed)


# The measured workloads (sizes and distributions of the solver's benchmark systems).
def system_2d_small():
    """32x32 interior nodes (n = 1024), sigma = 1.0, x_true ~ U(-1,1) seed 0, tau 1e-10."""
    return fem2d(32, sigma=1.0, jitter=0.3, seed=0, x_seed=0)


def system_2d_large(g=1108):
    """1108x1108 interior nodes (n = 1,227,664), sigma = 2.0, random symmetric permutation
    from seed 1 then reverse Cuthill-McKee, tau 1e-8."""
    return fem2d(g, sigma=2.0, jitter=0.3, seed=0, perm_seed=1, rcm=True, x_seed=0)


def system_3d(g=128):
    """128^3 interior nodes (n = 2,097,152), Kuhn tetrahedra, sigma = 1.5, jitter 0.25h."""
    return fem3d(g, sigma=1.5, jitter=0.25, seed=0, x_seed=0)


def batch_sides(count=512, lo=45, hi=256, seed=3):
    """Grid sides log-uniform in [lo, hi] and sigmas log-uniform in [0.5, 2.5], seeded."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(math.log(lo), math.log(hi), count)).round().astype(int)
    sigmas = np.exp(rng.uniform(math.log(0.5), math.log(2.5), count))
    return sides, sigmas


def rcm(row_ptr, col_idx) -> np.ndarray:
    n = len(row_ptr) - 1
    perm = np.empty(n, np.int32)
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    check(lib.xplus_rcm(n, ptr(rp), ptr(ci), ptr(perm)))
    return perm


def rcm_device(row_ptr, col_idx, device=0):
    """xplus_rcm_device on the GPU: (perm as a numpy array, whether the GPU ordering ran)."""
    import torch
    dev = torch.device("cuda", device)
    rp = torch.as_tensor(np.ascontiguousarray(row_ptr, np.int32), device=dev)
    ci = torch.as_tensor(np.ascontiguousarray(col_idx, np.int32), device=dev)
    n = len(row_ptr) - 1
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    used = C.c_int()
    torch.cuda.synchronize(dev)
    check(lib.xplus_rcm_device(n, rp.data_ptr(), ci.data_ptr(), perm.data_ptr(), C.byref(used), None))
    return perm.cpu().numpy(), bool(used.value)


def permute_symmetric_device(row_ptr, col_idx, values, perm, device=0):
    """xplus_permute_symmetric_device on the GPU; returns numpy arrays."""
    import torch
    dev = torch.device("cuda", device)
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dt), device=dev)  # noqa: E731
    rp, ci, v, pm = t(row_ptr, np.int32), t(col_idx, np.int32), t(values, np.float64), t(perm, np.int32)
    n = len(row_ptr) - 1
    orp = torch.empty(n + 1, dtype=torch.int32, device=dev)
    oci = torch.empty(len(col_idx), dtype=torch.int32, device=dev)
    ov = torch.empty(len(col_idx), dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    check(lib.xplus_permute_symmetric_device(n, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), pm.data_ptr(),
                                             orp.data_ptr(), oci.data_ptr(), ov.data_ptr(), None))
    return orp.cpu().numpy(), oci.cpu().numpy(), ov.cpu().numpy()


def permute_symmetric(row_ptr, col_idx, values, perm):
    n = len(row_ptr) - 1
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    pm = np.ascontiguousarray(perm, np.int32)
    orp = np.empty(n + 1, np.int32)
    oci = np.empty(len(ci), np.int32)
    ov = np.empty(len(ci), np.float64)
    check(lib.xplus_permute_symmetric(n, ptr(rp), ptr(ci), ptr(v), ptr(pm), ptr(orp), ptr(oci), ptr(ov)))
    return orp, oci, ov


def sell_build(row_ptr, col_idx, values, C_=32, sigma=256, chunk=1, diag_split=False) -> dict:
    n = len(row_ptr) - 1
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    v = np.ascontiguousarray(values, np.float64)
    ns, slots = C.c_int(), C.c_int64()
    args = (n, ptr(rp), ptr(ci), ptr(v), C_, sigma, chunk, int(diag_split))
    check(lib.xplus_sell_build(*args, C.byref(ns), C.byref(slots), None, None, None, None, None, None))
    perm = np.empty(n, np.int32)
    sp = np.empty(ns.value + 1, np.int64)
    sw = np.empty(ns.value, np.int32)
    col = np.empty(slots.value, np.int32)
    val = np.empty(slots.value, np.float64)
    diag = np.empty(n, np.float64) if diag_split else None
    check(lib.xplus_sell_build(*args, C.byref(ns), C.byref(slots), ptr(perm), ptr(sp), ptr(sw),
                               ptr(col), ptr(val), ptr(diag)))
    return dict(n_slices=ns.value, slots=slots.value, perm=perm, slice_ptr=sp, slice_width=sw,
                col=col, val=val, diag=diag)


def sell_build_device(row_ptr, col_idx, values, C_=32, sigma=256, chunk=1, diag_split=False, device=0) -> dict:
    """xplus_sell_build_device on torch CUDA tensors; returns the same fields as sell_build
    (as torch tensors on the device)."""
    import torch
    dev = torch.device("cuda", device)
    rp = torch.as_tensor(np.ascontiguousarray(row_ptr, np.int32), device=dev)
    ci = torch.as_tensor(np.ascontiguousarray(col_idx, np.int32), device=dev)
    v = torch.as_tensor(np.ascontiguousarray(values, np.float64), device=dev)
    n = len(row_ptr) - 1
    ns, slots = C.c_int(), C.c_int64()
    torch.cuda.synchronize(dev)
    args = (n, rp.data_ptr(), ci.data_ptr(), v.data_ptr(), C_, sigma, chunk, int(diag_split))
    check(lib.xplus_sell_build_device(*args, C.byref(ns), C.byref(slots), None, None, None, None, None, None, None))
    perm = torch.empty(n, dtype=torch.int32, device=dev)
    sp = torch.empty(ns.value + 1, dtype=torch.int64, device=dev)
    sw = torch.empty(ns.value, dtype=torch.int32, device=dev)
    col = torch.empty(slots.value, dtype=torch.int32, device=dev)
    val = torch.empty(slots.value, dtype=torch.float64, device=dev)
    diag = torch.empty(n, dtype=torch.float64, device=dev) if diag_split else None
    check(lib.xplus_sell_build_device(*args, C.byref(ns), C.byref(slots), perm.data_ptr(), sp.data_ptr(), sw.data_ptr(),
                                      col.data_ptr(), val.data_ptr(), None if diag is None else diag.data_ptr(), None))
    return dict(n_slices=ns.value, slots=slots.value, perm=perm, slice_ptr=sp, slice_width=sw, col=col, val=val,
                diag=diag)


def cuper_unpack(n, batch_count, sp_element_list_ptr, words, channel_words):
    """Decodes the reference's packed 16-channel words into COO (row, col, fp32 value)."""
    ptr_a = np.ascontiguousarray(sp_element_list_ptr, np.int32)
    w = np.ascontiguousarray(words, np.uint64)
    cnt = C.c_int64()
    check(lib.xplus_cuper_unpack(n, batch_count, ptr(ptr_a), ptr(w), int(channel_words), C.byref(cnt),
                                 None, None, None))
    rows = np.empty(cnt.value, np.int32)
    cols = np.empty(cnt.value, np.int32)
    vals = np.empty(cnt.value, np.float32)
    check(lib.xplus_cuper_unpack(n, batch_count, ptr(ptr_a), ptr(w), int(channel_words), C.byref(cnt),
                                 ptr(rows), ptr(cols), ptr(vals)))
    return rows, cols, vals
