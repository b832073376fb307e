"""ctypes binding of libfmma_b200.so (the C ABI declared in include/fmma_b200.h).

The library is built in-tree (``python -m fmma_b200.build``).  Importing this
module fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfmma_b200.so")

OK = 0
ERR_INVALID_ARG = 1
ERR_UNSUPPORTED_SOLVER = 2
ERR_OOM = 3
ERR_CUDA = 4
ERR_TIMEOUT = 5
ERR_NO_DEVICE = 6

KERNEL_INV_R = 0
KERNEL_INV_R_SAFE = 1
KERNEL_INV_DIFF = 2
KERNEL_LOG_R = 3
KERNEL_GAUSSIAN = 4
KERNEL_MULTIQUADRIC = 5
KERNEL_SUM_OVER_R2 = 6
KERNEL_SUM2_OVER_R2 = 7

SOLVER_EXACT = 0
SOLVER_FMM = 1
SOLVER_TREE = 2
SOLVER_NRNMM = 3

PREC_FP64 = 0
PREC_MIXED_TF32X3 = 1
PREC_MIXED_BF16X3 = 2

MEM_HOST = 0
MEM_DEVICE = 1

NUM_STAGES = 9

_i = C.c_int
_i64 = C.c_int64
_d = C.c_double
_vp = C.c_void_p
_pi = C.POINTER(C.c_int)
_pi64 = C.POINTER(C.c_int64)
_pd = C.POINTER(C.c_double)

# device allocator callbacks of fmma_set_allocator
ALLOC_FN = C.CFUNCTYPE(C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p)
FREE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p)

# name -> (restype, argtypes); every symbol declared in include/fmma_b200.h
SIGNATURES = {
    "fmma_ctx_create": (_i, [_i, C.POINTER(_vp)]),
    "fmma_ctx_destroy": (_i, [_vp]),
    "fmma_last_error": (C.c_char_p, []),
    "fmma_version": (C.c_char_p, []),
    "fmma_set_kernel": (_i, [_vp, _i, _d]),
    "fmma_set_allocator": (_i, [_vp, _vp, _vp, _vp]),
    "fmma_debug_m2l_wait": (_i, [_vp, C.c_longlong, _i]),
    "fmma_set_m2l_options": (_i, [_vp, _i, _i, _i, _i]),
    "fmma_set_schedule_options": (_i, [_vp, _i, _i]),
    "fmma_default_depth": (_i, [_i64, _i]),
    "fmma_solve_d": (_i, [_vp, _i, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_solve_f": (_i, [_vp, _i, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_solve_d1": (_i, [_vp, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_solve_d2": (_i, [_vp, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_solve_d3": (_i, [_vp, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_solve_f1": (_i, [_vp, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_solve_f2": (_i, [_vp, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_solve_f3": (_i, [_vp, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i, _pi]),
    "fmma_exact_rows_d": (_i, [_vp, _i, _i64, _vp, _i64, _vp, _i64, _vp, _i, _vp, _vp, _i]),
    "fmma_tree_export_d": (_i, [_vp, _i, _i, _i64, _vp, _i64, _vp, _vp, _vp, _vp, _i]),
    "fmma_interaction_list": (_i, [_vp, _i, _i64, _pi64, _i, _pi]),
    "fmma_near_list": (_i, [_vp, _i64, _pi64, _i, _pi]),
    "fmma_max_leaf_occupancy_d": (_i, [_vp, _i, _i, _i64, _vp, _i64, _vp, _i, _pi64, _pi64]),
    "fmma_stage_times": (_i, [_vp, _pd, _i]),
    "fmma_stage_name": (C.c_char_p, [_i]),
    "fmma_last_launch_count": (_i64, [_vp]),
    "fmma_ctx_stream": (_vp, [_vp]),
    "fmma_m2l_stats": (_i, [_vp, _pd, _pd, _pi64]),
    "fmma_tree_stats": (_i, [_vp, _pi64, _pi64, _pi64]),
    "fmma_set_user_kernel": (_i, [_vp, _vp, _vp, _i]),
    "fmma_exact_noalloc_d": (_i, [_i, _i, _d, _i64, _vp, _i64, _vp, _i, _vp, _vp, _vp]),
    "fmma_tree_levels": (_i, [_vp, _i, _pi, _vp, _vp]),
    "fmma_set_kernel_expr": (_i, [_vp, C.c_char_p, _i]),
    "fmma_solve_grad_d": (_i, [_vp, _i, _i, _i, _i, _i, _i, _i64, _vp, _i64, _vp, _i, _vp, _vp, _vp, _i, _pi]),
    "fmma_forest_solve_d": (_i, [_vp, _i, _i, _pi64, _vp, _pi64, _vp, _i, _vp, _vp, _i, _pi, _i, _i, _i]),
    "fmma_forest_depths_d": (_i, [_vp, _i, _i, _pi64, _vp, _pi64, _vp, _i, _i, _pi]),
    "fmma_plan_create_d": (_i, [_vp, _i, _i, _pi64, _vp, _pi64, _vp, _i, _i, _pi, _i, _i, _i, _i, C.POINTER(_vp)]),
    "fmma_plan_execute_d": (_i, [_vp, _vp, _vp, _i]),
    "fmma_plan_stats": (_i, [_vp, _pd, _pd, _pi, _pi, _pi64]),
    "fmma_plan_destroy": (_i, [_vp]),
    "fmma_set_tuner_cache": (_i, [_vp, C.c_char_p]),
    "fmma_cheb_nodes": (_i, [_i, _pd]),
    "fmma_cheb_fit_d": (_i, [_vp, _i, _i, _i, _vp, _vp, _i]),
    "fmma_cheb_eval_d": (_i, [_vp, _i, _i, _i, _vp, _i64, _vp, _vp, _i]),
}

_lib = None


class FmmaError(RuntimeError):
    """A non-OK status from the C ABI."""

    def __init__(self, status: int, message: str):
        super().__init__(f"fmma_b200 error {status}: {message}")
        self.status = status


def load() -> C.CDLL:
    """Loads libfmma_b200.so (once); raises ImportError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m fmma_b200.build` "
            "(the GPU path has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != OK:
        msg = load().fmma_last_error().decode(errors="replace")
        raise FmmaError(status, msg)
