"""ctypes access to the oracle (TEST INFRASTRUCTURE ONLY).

  C  = liboracle.so       the C restatement in pcg_oracle.c (always buildable with gcc)
  REF = _ref/libxplus_ref.so  the reference's own sources compiled by oracle/Makefile
                           (present when the reference tree was available at build time)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
C_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libxplus_ref.so"
# the reference's multi-kernel host program relinked against libxplus_b200.so, and the same
# program with the reference's own CPU kernels (oracle/Makefile relink)
RELINKED_HOST = HERE / "_ref" / "xplus_host_b200"
REFERENCE_HOST = HERE / "_ref" / "xplus_host_ref"


def reference_tree() -> Path | None:
    """The reference tree to compile from: $XPLUS_REFERENCE_TREE (it must hold the reference's
    src/), or None when the variable is unset (then no _ref build).  Only the build step reads
    the tree: tests and benchmarks load the prebuilt _ref library."""
    env = os.environ.get("XPLUS_REFERENCE_TREE")
    if not env:
        return None
    if not (Path(env) / "src").is_dir():
        raise FileNotFoundError(f"XPLUS_REFERENCE_TREE={env} does not hold the reference's src/")
    return Path(env)


def build(ref: bool = True) -> None:
    """Compiles liboracle.so, and the reference library when a reference tree is available."""
    subprocess.run(["make", "-s", "-C", str(HERE), "all"], check=True)
    tree = reference_tree() if ref else None
    if tree is not None:
        subprocess.run(["make", "-s", "-C", str(HERE), f"REF={tree}", "ref"], check=True)
        if (HERE.parent / "project_xplus_b200" / "lib" / "libxplus_b200.so").exists():
            subprocess.run(["make", "-s", "-C", str(HERE), f"REF={tree}", "relink"], check=True)


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


_c = None
_r = None


def clib():
    global _c
    if _c is None:
        if not C_LIB.exists():
            build(ref=False)
        _c = C.CDLL(str(C_LIB))
        _c.or_residual_norm.restype = C.c_double
    return _c


def reflib():
    """The reference built from source, or None when it was never built here."""
    global _r
    if _r is None and REF_LIB.exists():
        _r = C.CDLL(str(REF_LIB))
        _r.ref_last_error.restype = C.c_char_p
        _r.ref_cuper_last_error.restype = C.c_char_p
    return _r


def _csr(ds):
    return (np.ascontiguousarray(ds.row_ptr, np.int32), np.ascontiguousarray(ds.col_idx, np.int32),
            np.ascontiguousarray(ds.values, np.float64))


def golden(ds, tau, max_iters=0, x0=None, b=None, use_ref=False):
    """run_jacobi_pcg (src/CgSolverGolden.hpp:42).  Returns dict(x, iterations, final_rr,
    converged, trace[k, 5]); use_ref=True runs the reference's own code instead."""
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    b = np.ascontiguousarray(ds.b if b is None else b, np.float64)
    x0 = np.ascontiguousarray(ds.x0 if x0 is None else x0, np.float64)
    eff = max_iters if max_iters > 0 else max(4 * n, 1000)
    x = np.empty(n)
    tr = np.zeros((eff, 5))
    it, conv = C.c_int(), C.c_int()
    frr = C.c_double()
    if use_ref:
        lib = reflib()
        res = C.c_double()
        rc = lib.ref_golden(n, _p(rp), _p(ci), _p(v), _p(b), _p(x0), C.c_double(tau), int(max_iters),
                            _p(x), C.byref(it), C.byref(frr), C.byref(conv), _p(tr), C.byref(res))
        if rc:
            raise RuntimeError(lib.ref_last_error().decode())
    else:
        rc = clib().or_golden_pcg(n, _p(rp), _p(ci), _p(v), _p(b), _p(x0), C.c_double(tau), int(max_iters),
                                  _p(x), C.byref(it), C.byref(frr), C.byref(conv), _p(tr))
        if rc == 1:
            raise RuntimeError("breakdown: p^T A p is too small")
        if rc == 2:
            raise RuntimeError("tau must be positive")
        if rc == 3:
            raise RuntimeError("missing or zero diagonal entry")
    return dict(x=x, iterations=it.value, final_rr=frr.value, converged=bool(conv.value),
                trace=tr[:it.value].copy())


def multi_kernel(ds, tau, max_iters=0, use_ref=False):
    """run_local_multi_kernel_solver (archived/host/multi_kernel_solver.hpp:100).  The
    reference version keeps its n <= 1024 guard; the restatement has none."""
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    b = np.ascontiguousarray(ds.b, np.float64)
    x0 = np.ascontiguousarray(ds.x0, np.float64)
    eff = max_iters if max_iters > 0 else max(4 * n, 1000)
    x = np.empty(n)
    tr = np.zeros((eff, 5))
    it, st = C.c_int(), C.c_int()
    frr, res = C.c_double(), C.c_double()
    if use_ref:
        lib = reflib()
        rc = lib.ref_multi_kernel(n, _p(rp), _p(ci), _p(v), _p(b), _p(x0), C.c_double(tau), int(max_iters),
                                  _p(x), C.byref(it), C.byref(frr), C.byref(st), C.byref(res), _p(tr))
        if rc:
            raise RuntimeError(lib.ref_last_error().decode())
    else:
        rc = clib().or_multi_kernel_pcg(n, _p(rp), _p(ci), _p(v), _p(b), _p(x0), C.c_double(tau),
                                        int(max_iters), _p(x), C.byref(it), C.byref(frr), C.byref(st),
                                        C.byref(res), _p(tr))
        if rc:
            raise RuntimeError(f"multi-kernel oracle error {rc}")
    return dict(x=x, iterations=it.value, final_rr=frr.value, status=st.value, residual_l2=res.value,
                trace=tr[:it.value].copy())


def control(ds, tau, max_iters=0, spmv_mode=0):
    """cuper_pcg_control_kernel control flow (kernels/cuper_pcg_control_kernel.cpp:1069-1235),
    restated: spmv_mode 0 = FP64 SpMV, 1 = FP32 SpMV."""
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    eff = max_iters if max_iters > 0 else max(4 * n, 1000)
    minv = np.empty(n)
    assert clib().or_jacobi_inverse(n, _p(rp), _p(ci), _p(v), _p(minv)) == 0
    x = np.ascontiguousarray(ds.x0, np.float64).copy()
    r, z, p, ap = (np.zeros(n) for _ in range(4))
    met = np.zeros(4)
    st = np.zeros(2, np.int32)
    tr = np.zeros((eff, 5))
    b = np.ascontiguousarray(ds.b, np.float64)
    clib().or_control_pcg(n, _p(rp), _p(ci), _p(v), _p(b), _p(minv), _p(x), _p(r), _p(z), _p(p), _p(ap),
                          _p(met), _p(st), C.c_double(tau), eff, spmv_mode, _p(tr))
    return dict(x=x, metrics=met, status=int(st[0]), iterations=int(st[1]), trace=tr[:int(st[1])].copy())


def control_f32(ds, tau, max_iters):
    """Control-kernel algorithm at FP32 storage precision (values and vectors), FP64 dots."""
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    x = np.empty(n)
    st = np.zeros(2, np.int32)
    tr = np.zeros((max_iters, 5))
    b = np.ascontiguousarray(ds.b, np.float64)
    clib().or_control_pcg_f32(n, _p(rp), _p(ci), _p(v), _p(b), C.c_double(tau), int(max_iters), _p(x),
                              _p(st), _p(tr))
    return dict(x=x, status=int(st[0]), iterations=int(st[1]), trace=tr[:int(st[1])].copy())


def control_ref(ds, tau, max_iters=0):
    """The reference's own cuper_pcg_control_kernel compiled as C++ (packed 16-channel SpMV)."""
    lib = reflib()
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    x = np.empty(n)
    met = np.zeros(4)
    st = np.zeros(2, np.int32)
    b = np.ascontiguousarray(ds.b, np.float64)
    x0 = np.ascontiguousarray(ds.x0, np.float64)
    rc = lib.ref_control_solve(n, _p(rp), _p(ci), _p(v), _p(b), _p(x0), C.c_double(tau), int(max_iters),
                               _p(x), _p(met), _p(st))
    if rc:
        raise RuntimeError(lib.ref_cuper_last_error().decode())
    return dict(x=x, metrics=met, status=int(st[0]), iterations=int(st[1]))


def cuper_pcg_ref(ds, tau, max_iters=0):
    """run_cuper_pcg_solver (host/cuper_pcg_solver.hpp:311), the reference's own code."""
    lib = reflib()
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    x = np.empty(n)
    it, st = C.c_int(), C.c_int()
    frr, res = C.c_double(), C.c_double()
    tm = np.zeros(3)
    b = np.ascontiguousarray(ds.b, np.float64)
    x0 = np.ascontiguousarray(ds.x0, np.float64)
    rc = lib.ref_cuper_pcg(n, _p(rp), _p(ci), _p(v), _p(b), _p(x0), C.c_double(tau), int(max_iters), _p(x),
                           C.byref(it), C.byref(frr), C.byref(st), C.byref(res), _p(tm))
    if rc:
        raise RuntimeError(lib.ref_cuper_last_error().decode())
    return dict(x=x, iterations=it.value, final_rr=frr.value, status=st.value, residual_l2=res.value,
                plan_ms=tm[0], spmv_ms=tm[1], spmv_calls=int(tm[2]))


def spmv(ds, x):
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    y = np.empty(n)
    clib().or_spmv_csr(n, _p(rp), _p(ci), _p(v), _p(np.ascontiguousarray(x, np.float64)), _p(y))
    return y


def cuper_spmv(ds, x, use_ref=False):
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    y = np.empty(n)
    xx = np.ascontiguousarray(x, np.float64)
    if use_ref:
        assert reflib().ref_cuper_spmv(n, _p(rp), _p(ci), _p(v), _p(xx), _p(y)) == 0
    else:
        clib().or_cuper_style_spmv(n, _p(rp), _p(ci), _p(v), _p(xx), _p(y))
    return y


def residual_norm(ds, x, b=None):
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    bb = np.ascontiguousarray(ds.b if b is None else b, np.float64)
    return clib().or_residual_norm(n, _p(rp), _p(ci), _p(v), _p(bb), _p(np.ascontiguousarray(x, np.float64)))


def cuper_pack_ref(ds):
    """build_cuper_control_matrix (host/cuper_control_matrix.hpp:130), the reference's code."""
    lib = reflib()
    rp, ci, v = _csr(ds)
    n = len(rp) - 1
    bc, ml, cw = C.c_int(), C.c_int(), C.c_int()
    assert lib.ref_cuper_pack(n, _p(rp), _p(ci), _p(v), C.byref(bc), C.byref(ml), C.byref(cw), None, None) == 0
    ptr = np.empty(bc.value + 1, np.int32)
    words = np.empty(16 * cw.value, np.uint64)
    assert lib.ref_cuper_pack(n, _p(rp), _p(ci), _p(v), C.byref(bc), C.byref(ml), C.byref(cw), _p(ptr),
                              _p(words)) == 0
    return dict(batch_count=bc.value, matrix_len=ml.value, channel_words=cw.value, ptr=ptr, words=words)
