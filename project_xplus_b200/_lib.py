"""ctypes binding of libxplus_b200.so (the C ABI declared in include/xplus_b200.h).

The library is required: importing this module raises if it is missing, and every
compute entry point reports XPLUS_ERR_CUDA when no sm_100 GPU is present.  There is no
Python or CPU fallback for any solver operation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libxplus_b200.so"

XPLUS_CONVERGED, XPLUS_MAX_ITER, XPLUS_BREAKDOWN, XPLUS_TIMEOUT = 0, 1, 2, 3
XPLUS_OK, XPLUS_ERR_ARG, XPLUS_ERR_CUDA, XPLUS_ERR_DATA, XPLUS_ERR_IO, XPLUS_ERR_NOMEM = 0, 10, 11, 12, 13, 14
XPLUS_F32, XPLUS_BF16, XPLUS_F64, XPLUS_F16 = 0, 1, 2, 3
XPLUS_TAU_ABS_RR, XPLUS_TAU_REL_TRUE = 0, 1
XPLUS_NOALLOC_MAX_N = 4194304

STATUS_NAMES = {0: "converged", 1: "max_iter", 2: "breakdown", 3: "timeout"}
XPLUS_GNN_LOSS_PROBE = 0
XPLUS_GNN_LOSS_KAPORIN = 1


class XplusOpts(C.Structure):
    _fields_ = [
        ("value_type", C.c_int), ("vector_type", C.c_int), ("slice_height", C.c_int),
        ("sigma", C.c_int), ("chunk", C.c_int), ("keep_fp64", C.c_int),
        ("replace_every", C.c_int), ("replace_drop", C.c_double), ("block_threads", C.c_int),
        ("blocks_per_sm", C.c_int), ("barrier_timeout_s", C.c_double), ("device", C.c_int),
        ("row_sum_form", C.c_int), ("index16", C.c_int), ("l2_persist", C.c_int),
        ("resident", C.c_int), ("restart_on_replace", C.c_int), ("barriers_per_iter", C.c_int),
        ("stagnation_gain", C.c_double), ("stagnation_window", C.c_int), ("build_on_gpu", C.c_int),
        ("split_ratio", C.c_double),
    ]


class XplusMetrics(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("iterations", C.c_int), ("replacements", C.c_int),
        ("reserved0", C.c_int), ("rz", C.c_double), ("rr", C.c_double), ("pap", C.c_double),
        ("alpha", C.c_double), ("true_rel_residual", C.c_double), ("kernel_ms", C.c_double),
        ("setup_ms", C.c_double), ("reserved", C.c_double * 4),
    ]


class XplusError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


if not LIB_PATH.exists():
    raise ImportError(f"native library missing: {LIB_PATH} (run project_xplus_b200/build.py)")

lib = C.CDLL(str(LIB_PATH))

_p = C.c_void_p
_i = C.c_int
_d = C.c_double
_i64 = C.c_int64
_u64 = C.c_uint64
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

_SIGS = {
    "xplus_opts_default": (None, [C.POINTER(XplusOpts)]),
    "xplus_last_error_string": (C.c_char_p, []),
    "xplus_version": (C.c_char_p, []),
    "xplus_device_count": (_i, []),
    "xplus_pcg_create": (_i, [_p, _p, _p, _i, C.POINTER(XplusOpts), C.POINTER(_p)]),
    "xplus_pcg_destroy": (_i, [_p]),
    "xplus_pcg_solve": (_i, [_p, _p, _p, _d, _i, _i, _p, _ip, _p, _i, C.POINTER(XplusMetrics)]),
    "xplus_pcg_solve_device": (_i, [_p, _p, _p, _d, _i, _i, _p]),
    "xplus_pcg_last_metrics": (_i, [_p, C.POINTER(XplusMetrics)]),
    "xplus_pcg_last_trace": (_i, [_p, _p, _i]),
    "xplus_pcg_debug_skip_arrival": (_i, [_p, _i]),
    "xplus_pcg_last_phase_times": (_i, [_p, _p]),
    "xplus_pcg_last_block_times": (_i, [_p, _p, _i, _ip]),
    "xplus_pcg_spmv": (_i, [_p, _p, _p]),
    "xplus_pcg_spmv_device": (_i, [_p, _p, _p, _p]),
    "xplus_pcg_info": (_i, [_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64)]),
    "xplus_pcg_scratch_vectors": (_i, [_p, C.POINTER(_p), C.POINTER(_p)]),
    "xplus_pcg_control": (_i, [_p, _p, _p, _p, _p, _p, _p, _p, _p, _p, _d, _i, _i, _p]),
    "xplus_dataset_load_text": (_i, [C.c_char_p, _ip, _ip, _p, _p, _p, _p, _p]),
    "xplus_dataset_save_binary": (_i, [C.c_char_p, _i, _i, _p, _p, _p, _p, _p]),
    "xplus_dataset_load_binary": (_i, [C.c_char_p, _ip, _ip, _p, _p, _p, _p, _p]),
    "xplus_jacobi_diag": (_i, [_i, _p, _p, _p, _p]),
    "xplus_gen_fem2d": (_i, [_i, _d, _d, _u64, _i64, _i, _u64, _ip, _ip, _p, _p, _p, _p, _p]),
    "xplus_gen_fem3d": (_i, [_i, _d, _d, _u64, _i64, _i, _u64, _ip, _ip, _p, _p, _p, _p, _p]),
    "xplus_rcm": (_i, [_i, _p, _p, _p]),
    "xplus_rcm_device": (_i, [_i, _p, _p, _p, _ip, _p]),
    "xplus_permute_symmetric_device": (_i, [_i, _p, _p, _p, _p, _p, _p, _p, _p]),
    "xplus_permute_symmetric": (_i, [_i, _p, _p, _p, _p, _p, _p, _p]),
    "xplus_sell_build": (_i, [_i, _p, _p, _p, _i, _i, _i, _i, _ip, C.POINTER(_i64), _p, _p, _p, _p, _p, _p]),
    "xplus_sell_build_device": (_i, [_i, _p, _p, _p, _i, _i, _i, _i, _ip, C.POINTER(_i64), _p, _p, _p, _p, _p, _p, _p]),
    "xplus_cuper_unpack": (_i, [_i, _i, _p, _p, _i64, C.POINTER(_i64), _p, _p, _p]),
    "spmv_csr_kernel": (None, [_p, _p, _p, _p, _p, _i]),
    "spmv_blocked_kernel": (None, [_p, _p, _p, _p, _p, _i]),
    "init_pcg_kernel": (None, [_p, _p, _p, _p, _p, _p, _p, _i]),
    "dot_kernel": (None, [_p, _p, _p, _i]),
    "update_xrz_kernel": (None, [_p, _p, _p, _p, _p, _p, _p, _d, _i]),
    "update_p_kernel": (None, [_p, _p, _d, _i]),
    "xplus_update_xrz_noalloc": (_i, [_p, _p, _p, _p, _p, _p, _p, _d, _i, _p]),
    "xplus_pcg_set_gtg": (_i, [_p, _p, _p, _p, _i]),
    "xplus_pcg_set_gnn": (_i, [_p, _p, _p, _p, _p, _i, _dp]),
    "xplus_pcg_set_gnn_ex": (_i, [_p, _p, _p, _p, _p, _i, _i, _dp]),
    "xplus_pcg_get_gtg": (_i, [_p, _p, C.POINTER(_i64)]),
    "xplus_pcg_scale_gtg": (_i, [_p, _p, _p, _p]),
    "xplus_fsai_lower": (_i, [_i, _p, _p, _p, _p]),
    "xplus_gnn_param_count": (_i, []),
    "xplus_gnn_trainer_create": (_i, [_i, _p, _p, _p, _p, _i, _i, C.POINTER(_p)]),
    "xplus_gnn_trainer_destroy": (_i, [_p]),
    "xplus_gnn_set_params": (_i, [_p, _p]),
    "xplus_gnn_get_params": (_i, [_p, _p]),
    "xplus_gnn_loss_grad": (_i, [_p, _i, _u64, _dp, _p]),
    "xplus_gnn_set_loss": (_i, [_p, _i]),
    "xplus_gnn_adam": (_i, [_p, _p, _d]),
    "xplus_gnn_train": (_i, [_p, _i, _d, _d, _u64, _p]),
    "xplus_gnn_train_window": (_i, [_p, _i, _d, _d, _u64, _i64, _i64, _p]),
    "xplus_gnn_trainer_load": (_i, [_p, _i, _p, _p, _p, _p]),
    "xplus_gnn_predict": (_i, [_p, _i, _p, C.POINTER(_i64)]),
    "xplus_batch_create": (_i, [_i, _p, _p, _p, _p, C.POINTER(XplusOpts), C.POINTER(_p)]),
    "xplus_batch_destroy": (_i, [_p]),
    "xplus_batch_set_launch": (_i, [_p, _i, _i]),
    "xplus_batch_set_split": (_i, [_p, _i, _i, _i]),
    "xplus_batch_split_info": (_i, [_p, _ip, _ip, _ip, _ip]),
    "xplus_batch_set_resident": (_i, [_p, _i]),
    "xplus_batch_resident_info": (_i, [_p, _ip, _ip, _ip]),
    "xplus_batch_set_stage_matrix": (_i, [_p, _i]),
    "xplus_batch_staged_info": (_i, [_p, _ip, _ip, _ip]),
    "xplus_batch_autotune": (_i, [_p, _i, _d, _ip, _ip, _dp]),
    "xplus_batch_solve": (_i, [_p, _p, _p, _d, _i, _i, _p]),
    "xplus_batch_solve_device": (_i, [_p, _p, _p, _d, _i, _i, _p]),
    "xplus_batch_results": (_i, [_p, _p, _p, _p, _p, _p, _dp]),
    "xplus_batch_info": (_i, [_p, C.POINTER(_i64), C.POINTER(_i64), _ip, _ip, _ip, C.POINTER(_i64)]),
}

for _name, (_res, _args) in _SIGS.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

EXPORTED = tuple(_SIGS)


def last_error() -> str:
    s = lib.xplus_last_error_string()
    return s.decode() if s else ""


def check(rc: int) -> None:
    if rc != XPLUS_OK:
        raise XplusError(rc, last_error())


def default_opts(**kw) -> XplusOpts:
    o = XplusOpts()
    lib.xplus_opts_default(C.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o


def ptr(a) -> int | None:
    """Address of a numpy array or torch tensor (None passes NULL)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data
