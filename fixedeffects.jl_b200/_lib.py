"""ctypes binding of libfe_b200.so (include/fe_b200.h).

The library is the only compute path: importing this module without the
built library raises, and there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = _PKG / "libfe_b200.so"

FE_OK = 0
FE_ERR_INVALID = 1
FE_ERR_CUDA = 2
FE_ERR_ALLOC = 3
FE_ERR_TIMEOUT = 4

FE_PREC_FP64 = 0
FE_PREC_MIXED = 1
FE_PREC_FP32 = 2

FE_DTYPE_F64 = 0
FE_DTYPE_F32 = 1

FE_XCHG_F64 = 0
FE_XCHG_F32 = 1

# fe_exchange_fn: int (*)(void* ctx, void* buf, int64_t count, int32_t dtype, void* stream)
EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                               ctypes.c_int32, ctypes.c_void_p)

FE_OPT_TILE = 1
FE_OPT_CHECK_EVERY = 2
FE_OPT_MAX_ROUNDS = 3
FE_OPT_PROFILE = 4
FE_OPT_INNER_RHO = 5
FE_OPT_FUSE = 6
FE_OPT_EXPAND_VARIANT = 7
FE_OPT_SEGSUM_VARIANT = 8
FE_OPT_AUTOTUNE = 9
FE_OPT_MIXED_WARM_START = 10
FE_OPT_GRAPH = 11
FE_OPT_ROWSUM_VARIANT = 12
FE_OPT_ABSORB = 14
FE_OPT_FUSED_DEMEAN = 15
FE_OPT_ABSORB_SCALE = 16
FE_OPT_EXDM_PIPE = 17
FE_OPT_FIRM_ATOMIC = 18
FE_OPT_FUSED_RESID = 19

# every symbol declared in include/fe_b200.h
EXPORTS = (
    "fe_version", "fe_last_error", "fe_plan_create", "fe_plan_create_batch",
    "fe_plan_update_weights", "fe_plan_set_stream", "fe_plan_set_option",
    "fe_plan_destroy", "fe_solve_residuals", "fe_solve_residuals_device",
    "fe_solve_coefficients", "fe_plan_problem_results", "fe_plan_last_solve_info",
    "fe_plan_get_integer_plan", "fe_plan_get_scales", "fe_plan_primary",
    "fe_plan_kernel_stat", "fe_plan_reset_stats", "fe_plan_scales_noalloc",
    "fe_normalize_coefficients", "fe_full_coefficients", "fe_group_keys",
    "fe_solve_residuals_columns", "fe_plan_kernel_times", "fe_plan_create_sharded",
)

_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_f64p = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p
_vpp = ctypes.POINTER(ctypes.c_void_p)


class FEError(RuntimeError):
    """A non-zero status returned by the library."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[fe_b200 status {status}] {message}")
        self.status = status


_lib = None


def load(path: Path | str | None = None):
    """Loads libfe_b200.so and declares the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"{p} is missing: build it with `python fixedeffects.jl_b200/build.py` "
            "(the CUDA library is the only compute path)")
    L = ctypes.CDLL(str(p))
    sig = {
        "fe_version": (ctypes.c_int, []),
        "fe_last_error": (ctypes.c_char_p, []),
        "fe_plan_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int64, ctypes.c_int32,
                                          _vpp, _i64p, _vpp, _f64p, ctypes.c_int32]),
        "fe_plan_create_batch": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int32, _i64p,
                                                ctypes.c_int32, _vpp, _i64p, _vpp, _f64p,
                                                ctypes.c_int32]),
        "fe_plan_update_weights": (ctypes.c_int, [_vp, _f64p]),
        "fe_plan_set_stream": (ctypes.c_int, [_vp, _vp]),
        "fe_plan_set_option": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_double]),
        "fe_plan_destroy": (ctypes.c_int, [_vp]),
        "fe_solve_residuals": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int64,
                                              ctypes.c_int64, ctypes.c_int32, ctypes.c_double,
                                              ctypes.c_int64, _i64p, _u8p]),
        "fe_solve_residuals_device": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int64,
                                                     ctypes.c_int64, ctypes.c_int32,
                                                     ctypes.c_double, ctypes.c_int64, _i64p,
                                                     _u8p]),
        "fe_solve_coefficients": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_double, ctypes.c_int64, _vpp, _i64p,
                                                 _u8p]),
        "fe_plan_problem_results": (ctypes.c_int, [_vp, _i64p, _u8p]),
        "fe_plan_last_solve_info": (ctypes.c_int, [_vp, ctypes.c_int64, _f64p, _i32p, _i64p]),
        "fe_plan_get_integer_plan": (ctypes.c_int, [_vp, _i32p, _vpp, _vpp]),
        "fe_plan_get_scales": (ctypes.c_int, [_vp, _vpp]),
        "fe_plan_primary": (ctypes.c_int, [_vp, _i32p]),
        "fe_plan_kernel_stat": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_char_p,
                                               ctypes.c_int64, _i64p, _f64p, _f64p]),
        "fe_plan_reset_stats": (ctypes.c_int, [_vp]),
        "fe_plan_kernel_times": (ctypes.c_int, [_vp, ctypes.c_int32,
                                                ctypes.POINTER(ctypes.c_float), ctypes.c_int64,
                                                _i64p]),
        "fe_plan_scales_noalloc": (ctypes.c_int, [_vp, ctypes.c_int32, _vp, _vp]),
        "fe_normalize_coefficients": (ctypes.c_int, [_vp, _vpp, ctypes.c_int32]),
        "fe_full_coefficients": (ctypes.c_int, [_vp, _vpp, ctypes.c_int32, _vpp, ctypes.c_int32]),
        "fe_group_keys": (ctypes.c_int, [_vpp, ctypes.c_int32, ctypes.c_int64, ctypes.c_int32,
                                         _i64p, _i64p]),
        "fe_solve_residuals_columns": (ctypes.c_int, [_vp, _vpp, ctypes.c_int32, ctypes.c_int64,
                                                      ctypes.c_int32, ctypes.c_double,
                                                      ctypes.c_int64, _i64p, _u8p]),
        "fe_plan_create_sharded": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int64,
                                                  ctypes.c_int32, _vpp, _i64p, _vpp, _f64p,
                                                  ctypes.c_int32, EXCHANGE_FN, _vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def check(status: int) -> None:
    if status != FE_OK:
        msg = load().fe_last_error()
        raise FEError(status, msg.decode() if msg else "")
