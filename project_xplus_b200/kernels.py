"""The reference's multi-kernel ABI (archived/include/cg_kernels.hpp:9-54) run on the GPU.

Each function takes numpy arrays (staged to the device) or CUDA torch tensors (zero copy)
with the reference's argument order, and blocks until the outputs are written.  A call
that fails leaves its message in last_error() -- the reference's functions return void.
"""
from __future__ import annotations

from ._lib import last_error, lib, ptr  # noqa: F401


def spmv_csr_kernel(row_ptr, col_idx, values, x, y, n):
    lib.spmv_csr_kernel(ptr(row_ptr), ptr(col_idx), ptr(values), ptr(x), ptr(y), int(n))


def spmv_blocked_kernel(row_ptr, col_idx, values, x, y, n):
    lib.spmv_blocked_kernel(ptr(row_ptr), ptr(col_idx), ptr(values), ptr(x), ptr(y), int(n))


def init_pcg_kernel(b, ax, m_inv, r, z, p, metrics, n):
    lib.init_pcg_kernel(ptr(b), ptr(ax), ptr(m_inv), ptr(r), ptr(z), ptr(p), ptr(metrics), int(n))


def dot_kernel(a, b, out, n):
    lib.dot_kernel(ptr(a), ptr(b), ptr(out), int(n))


def update_xrz_kernel(x, p, r, ap, m_inv, z, metrics, alpha, n):
    lib.update_xrz_kernel(ptr(x), ptr(p), ptr(r), ptr(ap), ptr(m_inv), ptr(z), ptr(metrics), float(alpha), int(n))


def update_p_kernel(z, p, beta, n):
    lib.update_p_kernel(ptr(z), ptr(p), float(beta), int(n))
