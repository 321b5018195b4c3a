"""ctypes binding of libsmax_b200.so (the C ABI declared in include/smax_b200.h).

The library is built in-tree by ``python smaxkernels_b200/build.py`` (or
``__graft_entry__.build()``).  There is no fallback: if the library is missing
or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsmax_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is not built; run `python smaxkernels_b200/build.py`")

lib = C.CDLL(LIB_PATH)

P = C.c_void_p
U64 = C.c_uint64
I32 = C.c_int
PP = C.POINTER(C.c_void_p)
PU64 = C.POINTER(C.c_uint64)

# name -> (restype, argtypes); kept in the order of include/smax_b200.h
SIGNATURES = {
    "smax_abi_version": (I32, []),
    "smax_last_error": (C.c_char_p, []),
    "smax_test_fail_device_alloc": (I32, [C.c_int64]),
    "smax_test_device_alloc_count": (U64, []),
    "smax_ctx_create": (I32, [PP]),
    "smax_ctx_destroy": (I32, [P]),
    "smax_ctx_get_n_levels": (I32, [P]),
    "smax_ctx_get_level_ptr_at": (I32, [P, I32]),
    "smax_ctx_set_levels": (I32, [P, I32, P]),
    "smax_kernel_create": (I32, [PP, P, I32, I32, I32]),
    "smax_kernel_destroy": (I32, [P]),
    "smax_kernel_set_flag": (I32, [P, I32, I32]),
    "smax_kernel_register_A_crs": (I32, [P, U64, U64, U64, P, P, P]),
    "smax_kernel_register_A_scs": (I32, [P] + [U64] * 8 + [P] * 5),
    "smax_kernel_register_A_bcrs": (I32, [P] + [U64] * 7 + [P] * 3),
    "smax_kernel_register_B_crs": (I32, [P, U64, U64, U64, P, P, P]),
    "smax_kernel_register_C_crs_ref": (I32, [P, PU64, PU64, PU64, PP, PP, PP]),
    "smax_kernel_register_dense": (I32, [P, I32, U64, U64, P]),
    "smax_kernel_initialize": (I32, [P, U64, U64, U64]),
    "smax_kernel_apply": (I32, [P, U64, U64, U64]),
    "smax_kernel_finalize": (I32, [P, U64, U64, U64]),
    "smax_kernel_run": (I32, [P, U64, U64, U64]),
    "smax_kernel_sync": (I32, [P]),
    "smax_kernel_get_timer": (I32, [P, C.c_char_p, C.POINTER(C.c_double)]),
    "smax_kernel_stream": (P, [P]),
    "smax_kernel_swap_operands": (I32, [P]),
    "smax_kernel_set_stream": (I32, [P, P]),
    "smax_kernel_adjoint": (I32, [P, P, P, P, P]),
    "smax_kernel_update_A_values": (I32, [P, P]),
    "smax_kernel_get_refine_stats": (I32, [P, C.POINTER(I32), C.POINTER(C.c_double)]),
    "smax_kernel_autotune": (I32, [P, P]),
    "smax_utils_tune_spmv_format": (I32, [I32, U64, U64, U64, P, P, P, P]),
    "smax_batch_sptrsv_create": (I32, [PP, I32, I32, PU64, PU64, PP, PP, PP]),
    "smax_batch_sptrsv_solve": (I32, [P, P, P, I32, P]),
    "smax_batch_row_offset": (U64, [P, I32]),
    "smax_batch_info": (I32, [P, PU64, C.POINTER(I32), C.POINTER(I32)]),
    "smax_batch_destroy": (I32, [P]),
    "smax_utils_convert_crs_to_scs": (I32, [I32, I32, U64, U64, U64, P, P, P, U64, U64, PU64] + [PP] * 5),
    "smax_utils_convert_crs_to_bcrs": (I32, [I32, I32, U64, U64, U64, P, P, P, U64, U64, U64, U64, I32, PU64]
                                       + [PP] * 3),
    "smax_utils_build_symmetric_crs": (I32, [I32, U64, P, P, PP, PP, PU64]),
    "smax_utils_generate_perm": (I32, [P, I32, U64, P, P, P, P, C.c_char_p]),
    "smax_utils_sanity_check_perm": (I32, [I32, U64, P, P, P, C.POINTER(I32), C.POINTER(C.c_int64)]),
    "smax_utils_apply_mat_perm": (I32, [I32, I32, U64, P, P, P, P, P, P, P, P]),
    "smax_utils_apply_vec_perm": (I32, [I32, U64, P, P, P]),
    "smax_utils_read_mtx": (I32, [C.c_char_p, I32, PU64, PU64, PU64, PP, PP, PP]),
    "smax_utils_convert_coo_to_crs": (I32, [I32, U64, U64, U64, P, P, P, PP, PP, PP]),
    "smax_free_host": (None, [P]),
    "smax_spmv_crs_noalloc": (I32, [I32, U64, U64, U64, P, P, P, P, P, P]),
    "smax_measure_gather": (I32, [I32, I32, I32, I32, U64, P, P, P, U64, P, P, P]),
    "smax_solver_create": (I32, [PP, I32, I32, U64, U64, P, P, P]),
    "smax_solver_solve": (I32, [P, P, P, P, P, P]),
    "smax_solver_get_history": (I32, [P, P, I32, C.POINTER(I32)]),
    "smax_solver_destroy": (I32, [P]),
}



class Tuning(C.Structure):
    """struct smax_tuning"""
    _fields_ = [("spmv_variant", C.c_int), ("solve_mode", C.c_int), ("level_merge", C.c_int),
                ("sweep_cluster", C.c_int), ("from_cache", C.c_int), ("n_candidates", C.c_int),
                ("seconds", C.c_double)]


class FormatChoice(C.Structure):
    """struct smax_format_choice"""
    _fields_ = [("format", C.c_int), ("spmv_variant", C.c_int), ("C", C.c_int), ("sigma", C.c_int),
                ("b_height", C.c_int), ("b_width", C.c_int), ("n_candidates", C.c_int), ("seconds", C.c_double),
                ("crs_seconds", C.c_double)]


class SolverOpts(C.Structure):
    """struct smax_solver_opts"""
    _fields_ = [("tol", C.c_double), ("max_iters", C.c_int), ("check_length", C.c_int), ("mode", C.c_int)]


class SolverStats(C.Structure):
    """struct smax_solver_stats"""
    _fields_ = [("n_iters", C.c_int), ("converged", C.c_int), ("residual_norm", C.c_double),
                ("n_checks", C.c_int), ("host_waits", C.c_int)]


def struct_dict(s) -> dict:
    return {name: getattr(s, name) for name, _ in s._fields_}


for _name, (_res, _args) in SIGNATURES.items():
    _f = getattr(lib, _name)
    _f.restype = _res
    _f.argtypes = _args

# status codes (include/smax_b200.h)
OK = 0
ERR_BAD_ARG = -1
ERR_UNSUPPORTED_TYPE = -2
ERR_OOM = -3
ERR_ZERO_DIAG = -4
ERR_NO_DIAG = -5
ERR_TIMEOUT = -6
ERR_CUDA = -7
ERR_COL_OOB = -8
ERR_STATE = -9
ERR_UNSUPPORTED = -10

STATUS_NAMES = {0: "OK", -1: "BAD_ARG", -2: "UNSUPPORTED_TYPE", -3: "OOM", -4: "ZERO_DIAG", -5: "NO_DIAG",
                -6: "TIMEOUT", -7: "CUDA", -8: "COL_OOB", -9: "STATE", -10: "UNSUPPORTED"}


class SmaxError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{STATUS_NAMES.get(code, code)}] {msg}")
        self.code = code


def check(rc: int) -> int:
    if rc != OK:
        msg = lib.smax_last_error()
        raise SmaxError(rc, msg.decode() if msg else "")
    return rc
