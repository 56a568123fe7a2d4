"""ctypes binding of libpsipm_b200.so (declared in include/psipm_b200.h).

The shared library is built in-tree by ``make -C mf-psipm_b200`` (or
``__graft_entry__.build()``).  Importing this module never falls back to a
CPU implementation: if the library or a CUDA device is missing, the first
call raises ``GpuUnavailable``.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpsipm_b200.so")

OK = 0
ERR_ARGUMENT = -1
ERR_CUDA = -2
ERR_NOT_PD = -3
ERR_STATE = -4
ERR_BOUNDS = -5
ERR_TIMEOUT = -6
ERR_MEMORY = -7
ERR_SYMBOLIC = -8
ERR_UNSUPPORTED = -9

STATIC_SCRATCH_MAX = 1 << 20  # columns, psipm_normal_matvec_static
MLP_INPUTS = 6
MLP_WEIGHTS = 4608
MLP_BIASES = 130
MLP_PARAMS = 4738
MLP_TILE = 128

PCG_SPECTRAL = 0
PCG_HSD = 1
FP64 = 0
FP32_REFINED = 1
FP32_PRECOND = 2

STATUS_NAMES = {
    ERR_ARGUMENT: "invalid argument",
    ERR_CUDA: "CUDA error",
    ERR_NOT_PD: "not positive definite",
    ERR_STATE: "call order",
    ERR_BOUNDS: "device bounds check",
    ERR_TIMEOUT: "device deadline",
    ERR_MEMORY: "device memory",
    ERR_SYMBOLIC: "symbolic analysis",
    ERR_UNSUPPORTED: "unsupported",
}


class GpuUnavailable(RuntimeError):
    """The CUDA library or device is missing; there is no CPU fallback."""


class PcgInfo(ctypes.Structure):
    _fields_ = [
        ("info", ctypes.c_int32),
        ("iterations", ctypes.c_int32),
        ("matvecs", ctypes.c_int32),
        ("replacements", ctypes.c_int32),
        ("residual_checks", ctypes.c_int32),
        ("n_alpha", ctypes.c_int32),
        ("n_beta", ctypes.c_int32),
        ("n_history", ctypes.c_int32),
        ("refinements", ctypes.c_int32),
        ("ok", ctypes.c_int32),
        ("relative_residual", ctypes.c_double),
        ("seconds", ctypes.c_double),
        ("phase_seconds", ctypes.c_double * 4),
    ]


class FactorInfo(ctypes.Structure):
    _fields_ = [
        ("nsupernodes", ctypes.c_int32),
        ("nlevels", ctypes.c_int32),
        ("max_front", ctypes.c_int32),
        ("symbolic_analyses", ctypes.c_int32),
        ("nnz_factor", ctypes.c_int64),
        ("flops", ctypes.c_double),
        ("symbolic_seconds", ctypes.c_double),
        ("factor_seconds", ctypes.c_double),
    ]


_P = ctypes.c_void_p
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

SIGNATURES = {
    "psipm_create": (_I32, [_I64, _I64, _I64, _P, _P, _P, _I32, _I32, ctypes.POINTER(_P)]),
    "psipm_destroy": (None, [_P]),
    "psipm_last_error": (ctypes.c_char_p, [_P]),
    "psipm_set_low_rank": (_I32, [_P, _P, _I64]),
    "psipm_num_candidates": (_I64, [_P]),
    "psipm_get_candidates": (_I32, [_P, _P]),
    "psipm_set_theta": (_I32, [_P, _P, _D]),
    "psipm_scores": (_I32, [_P, _D, _P, _P]),
    "psipm_refresh_core": (_I32, [_P, _I64, _D, _I32, _P, _I64, _P, _P, _P]),
    "psipm_set_core": (_I32, [_P, _P, _I64]),
    "psipm_tie_info": (_I32, [_P, _P]),
    "psipm_set_grid": (_I32, [_P, _I32]),
    "psipm_set_deterministic": (_I32, [_P, _I32]),
    "psipm_set_factor_tc": (_I32, [_P, _I32]),
    "psipm_top_k": (_I32, [_P, _P, _I64, _P, _I64, _P, _P]),
    "psipm_factor": (_I32, [_P, _D, _I32, _P, _P]),
    "psipm_apply": (_I32, [_P, _P, _P]),
    "psipm_matvec": (_I32, [_P, _P, _P]),
    "psipm_pcg": (_I32, [_P, _P, _D, _I32, _I32, _I32, _D, _P, _P, _P, _P, _P, _P]),
    "psipm_set_pcg_budget": (_I32, [_P, _D]),
    "psipm_solve": (_I32, [_P, _P, _P, _D, _I32, _I32, _I32, _D, _P, _P, _P, _P, _P, _P, _P]),
    "psipm_solve_dev": (_I32, [_P, _P, _P, _D, _I32, _I32, _I32, _D, _P, _P, _P]),
    "psipm_kernel_launches": (_I64, [_P]),
    "psipm_set_profiling": (_I32, [_P, _I32]),
    "psipm_timer_start": (_I32, [_P]),
    "psipm_normal_matvec_static": (_I32, [_I64, _I64, _P, _P, _P, _P, _P, _P, _P, _D, _P, _P, _P]),
    "psipm_debug_apply_trace": (_I32, [_P, _P, _P, _P, _I32, _P, _P]),
    "psipm_timer_stop": (_I32, [_P, _P]),
    "psipm_debug_barrier_timeout": (_I32, [_P, _I32, _I32, _I32, _P]),
    "psipm_debug_syrk_tc": (_I32, [_I32, _I32, _I32, _I32, _I32, _I32, _P, _P]),
    "psipm_debug_levels": (_I32, [_P, _P, _I32, _P]),
    "psipm_ipm_load": (_I32, [_P, _P, _P, _P, _P, _P]),
    "psipm_ipm_put": (_I32, [_P, _I32, _P, _P, _P, _P]),
    "psipm_ipm_get": (_I32, [_P, _I32, _P, _P, _P, _P]),
    "psipm_ipm_copy": (_I32, [_P, _I32]),
    "psipm_ipm_residuals": (_I32, [_P, _D, _D, _P]),
    "psipm_ipm_theta": (_I32, [_P, _D, _D, _D]),
    "psipm_ipm_targets": (_I32, [_P, _I32, _P]),
    "psipm_ipm_newton": (_I32, [_P, _I32, _D, _I32, _I32, _I32, _D, _P, _P, _P, _P, _P]),
    "psipm_ipm_start_solve": (_I32, [_P, _I32, _D, _I32, _I32, _I32, _D, _P, _P, _P, _P, _P]),
    "psipm_ipm_start": (_I32, [_P, _I32, _P]),
    "psipm_ipm_steps": (_I32, [_P, _I32, _D, _P]),
    "psipm_ipm_complementarity": (_I32, [_P, _I32, _D, _D, _D, _P]),
    "psipm_ipm_accept": (_I32, [_P, _D]),
    "psipm_ipm_update": (_I32, [_P, _D, _D]),
    "psipm_ipm_metrics": (_I32, [_P, _P]),
    "psipm_lag_reference": (_I32, [_P]),
    "psipm_lag_ratio": (_I32, [_P, _P]),
    "psipm_minres": (_I32, [_P, _P, _P, _D, _I32, _D, _P, _P, _P]),
    "psipm_get_theta": (_I32, [_P, _P]),
    "psipm_set_tree": (_I32, [_P, _P, _P, _P]),
    "psipm_tree_factor": (_I32, [_P, _P, _D]),
    "psipm_tree_get": (_I32, [_P, _P, _P]),
    "psipm_price_load": (_I32, [_P, _P]),
    "psipm_price": (_I32, [_P, _P, _D, _P, _D, _I64, _P, _P, _P]),
    "psipm_mlp_features": (_I32, [_P, _D, _P]),
    "psipm_mlp_scores": (_I32, [_P, _P, _P, _D, _I64, _P]),
    "psipm_mlp_forward_dev": (_I32, [_I64, _P, _P, _P, _P, _P]),
    "psipm_mlp_grad_dev": (_I32, [_I64, _P, _P, ctypes.c_float, ctypes.c_float, _P, _P, _I32, _P, _P,
                                  ctypes.c_float, _P, _P, _P]),
    "psipm_mlp_adam_dev": (_I32, [_P, _P, _P, _P, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                  ctypes.c_float, _I32, ctypes.c_float, _P, _P, _P]),
    "psipm_ipm_minres": (_I32, [_P, _I32, _D, _I32, _D, _P, _P]),
}

_lib: Optional[ctypes.CDLL] = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the library once and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise GpuUnavailable(
            f"{path} is missing: build it with `make -C mf-psipm_b200` (nvcc, sm_100a)"
        )
    lib = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def i64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int64)
