"""project_xplus_b200 -- B200-native Jacobi-preconditioned CG, a drop-in for project-xplus's
PCG path.  The compute path is libxplus_b200.so (sm_100a kernels behind a C ABI,
include/xplus_b200.h); this package is its host-side mirror of the reference's solver entry.
"""
from . import _lib  # noqa: F401  (raises ImportError when the native library is missing)
from ._lib import (XPLUS_BF16, XPLUS_F16, XPLUS_F32, XPLUS_F64, XPLUS_TAU_ABS_RR, XPLUS_TAU_REL_TRUE,  # noqa: F401
                   XplusError)
from .solver import (CsrDataset, IterationTrace, PcgResult, PcgSolver, SolverConfig,  # noqa: F401
                     build_jacobi_inverse, device_count, log_iteration, run_defaults, run_pcg)

__all__ = ["CsrDataset", "PcgSolver", "PcgResult", "SolverConfig", "IterationTrace", "run_pcg",
           "run_defaults", "build_jacobi_inverse", "log_iteration", "device_count", "XplusError",
           "XPLUS_F32", "XPLUS_BF16", "XPLUS_F16", "XPLUS_F64", "XPLUS_TAU_ABS_RR", "XPLUS_TAU_REL_TRUE"]
