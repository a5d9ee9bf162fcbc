"""Loads libalgebra_linear_gpu.so and declares the C ABI of
include/algebra_linear_gpu.h for ctypes.

The library is the product; there is no CPU fallback. If the shared object is
missing, every import of this module raises.
"""

from __future__ import annotations

import ctypes as C
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libalgebra_linear_gpu.so"

# status codes (include/algebra_linear_gpu.h)
OK = 0
SINGULAR = 1
BAD_SHAPE = 2
CONVERGENCE = 3
NOT_IMPLEMENTED = 4
SP_BAD_SHAPE = 100
SP_INVALID_STRUCTURE = 101
SP_UNSORTED_ROWS = 102
SP_DUPLICATE_ENTRY = 103
SP_SINGULAR = 104
SP_INDEX_OVERFLOW = 105
SP_STRUCTURE_MISMATCH = 106
SP_NOT_FINITE = 107
SP_NOT_FACTORIZED = 108
CUDA_ERROR = 200
OUT_OF_DEVICE_MEMORY = 201
TIMEOUT = 202
INVALID_ARGUMENT = 203
NO_DEVICE = 204

KERNEL_CLASSES = ["panel", "laswp", "trsm", "gemm", "gemm_tc", "solve", "resid", "cast", "batch",
                  "sparse", "misc"]

UPDATE_EXACT = 0
UPDATE_FMA = 1

_P = C.c_void_p
_SZ = C.c_size_t
_I = C.c_int
_D = C.POINTER(C.c_double)
_SZP = C.POINTER(C.c_size_t)

# (name, restype, argtypes) for every declared entry point
SIGNATURES = [
    ("alg_status_string", C.c_char_p, [_I]),
    ("alg_version", C.c_char_p, []),
    ("alg_kernel_launch_count", C.c_ulonglong, []),
    ("alg_dgetrf", _I, [_P, _SZ, _P, _P]),
    ("alg_dgetrf_rect", _I, [_P, _SZ, _SZ, _P]),
    ("alg_dgesv", _I, [_P, _P, _SZ]),
    ("alg_dgetri", _I, [_P, _SZ, _P]),
    ("alg_zgetrf", _I, [_P, _SZ, _P]),
    ("alg_zgetrf_rect", _I, [_P, _SZ, _SZ, _P]),
    ("alg_zgesv", _I, [_P, _P, _SZ]),
    ("alg_zgetri", _I, [_P, _SZ, _P]),
    ("alg_dgesv_nrhs", _I, [_P, _P, _SZ, _SZ]),
    ("alg_dgesv_ex", _I, [_I, _P, _P, _SZ, _SZ, _P]),
    ("alg_ctx_create", _I, [_P, C.POINTER(_P)]),
    ("alg_ctx_destroy", None, [_P]),
    ("alg_ctx_set_stream", _I, [_P, _P]),
    ("alg_ctx_set_wait_limit", _I, [_P, C.c_ulonglong]),
    ("alg_ctx_inject_stuck_wait", _I, [_P, _I]),
    ("alg_dgetrf_dev", _I, [_P, _I, _P, _I, _I, _P, _P]),
    ("alg_dgetrf_rect_dev", _I, [_P, _I, _P, _I, _I, _I, _P]),
    ("alg_dgetrs_dev", _I, [_P, _P, _I, _I, _P, _P, _I, _I]),
    ("alg_dgetri_dev", _I, [_P, _P, _I, _I, _P]),
    ("alg_dgesv_dev", _I, [_P, _I, _P, _I, _I, _P, _I, _I, _P]),
    ("alg_larnv_dev", _I, [_P, _I, _P, _SZ, _P, _P]),
    ("alg_mixed_opts_default", None, [_P]),
    ("alg_dgesv_mixed", _I, [_P, _P, _P, _SZ, _SZ, _P]),
    ("alg_dgesv_mixed_dev", _I, [_P, _P, _P, _I, _I, _P, _I, _I, _P]),
    ("alg_batch_create", _I, [_P, _I, _P, _I, C.POINTER(_P)]),
    ("alg_batch_offsets", _I, [_P, _P, _P]),
    ("alg_batch_solve", _I, [_P, _P, _P, _P]),
    ("alg_batch_solve_graph", _I, [_P, _P, _P, _P]),
    ("alg_batch_autotune", _I, [_P, _P, _P, _P, _P, _P, _P]),
    ("alg_batch_info", _I, [_P, _P, _P, _P, _P, _P]),
    ("alg_batch_panels", _I, [_P, _P]),
    ("alg_batch_set_config", _I, [_P, _I, _I, _I]),
    ("alg_batch_eta", _I, [_P, _P]),
    ("alg_batch_ipiv", _I, [_P, _P]),
    ("alg_batch_destroy", None, [_P]),
    ("alg_gemm_tc_sub_dev", _I, [_P, _I, _I, _I, _I, _P, _I, _P, _I, _P, _I]),
    ("alg_gemm_dmma_sub_dev", _I, [_P, _I, _I, _I, _P, _I, _P, _I, _P, _I]),
    ("alg_dgesv_mixed_noalloc", _I, [_P, _P, _P, _I, _P, _P, _P]),
    ("alg_splu_analyze", _I, [_P, _SZ, _P, _SZ, _I, C.c_double, _P]),
    ("alg_splu_factorize", _I, [_P, _P, _SZ, _P, _SZ, _P, _SZ]),
    ("alg_splu_solve", _I, [_P, _P, _SZ]),
    ("alg_zsplu_factorize", _I, [_P, _P, _SZ, _P, _SZ, _P, _SZ]),
    ("alg_zsplu_solve", _I, [_P, _P, _SZ]),
    ("alg_splu_effective_method", _I, [_P]),
    ("alg_splu_flop_ratio", _I, [_P, _P]),
    ("alg_splu_get_stats", _I, [_P, _P]),
    ("alg_splu_free", None, [_P]),
    ("alg_splu_symbolic", _I, [_P, _P, _P, _P, _P, _P]),
    ("alg_splu_row_perm", _I, [_P, _P]),
    ("alg_splu_plan_info", _I, [_P, _P]),
    ("alg_splu_set_ctx", _I, [_P, _P]),
    ("alg_splu_factorize_dev", _I, [_P, _P]),
    ("alg_splu_solve_dev", _I, [_P, _P]),
    ("alg_splu_clone", _I, [_P, _P]),
    ("alg_splu_factorize_values", _I, [_P, _P]),
    ("alg_splu_set_precision", _I, [_P, _I, C.c_double, _I]),
    ("alg_splu_last_solve", _I, [_P, _P]),
    ("alg_server_create", _I, [_I, _SZ, _SZ, _P]),
    ("alg_server_submit", _I, [_P, _P]),
    ("alg_server_wait", _I, [_P, _P]),
    ("alg_server_drain", _I, [_P]),
    ("alg_server_completed", C.c_ulonglong, [_P]),
    ("alg_server_now_ns", C.c_int64, []),
    ("alg_server_destroy", None, [_P]),
    ("alg_ctx_set_profiling", _I, [_P, _I]),
    ("alg_ctx_profile_reset", _I, [_P]),
    ("alg_ctx_profile_get", _I, [_P, _I, C.POINTER(C.c_ulonglong), C.POINTER(C.c_double),
                                 C.POINTER(C.c_double), C.POINTER(C.c_double)]),
]

_lib = None


def load() -> C.CDLL:
    """Returns the loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH.name} is missing: build it with `python -m algebra_linear_b200.build`"
            )
        lib = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def status_string(code: int) -> str:
    return load().alg_status_string(code).decode()


def ptr(arr) -> int:
    """Address of a numpy array's data or a torch tensor's storage."""
    if hasattr(arr, "data_ptr"):
        return arr.data_ptr()
    return arr.ctypes.data
