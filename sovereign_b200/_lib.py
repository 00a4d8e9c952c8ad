"""Loader for libsovipm.so, the C-ABI engine (include/sov_ipm.h).

The library is built in-tree (``python -m sovereign_b200.build``) and loaded from
sovereign_b200/libsovipm.so. There is no CPU fallback: a missing library or a missing sm_100
device raises.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsovipm.so")

# every symbol include/sov_ipm.h declares
EXPORTS = [
    "sov_default_lp_options", "sov_default_qp_options", "sov_ipm_dims", "sov_lp_solve", "sov_qp_solve",
    "sov_lp_solve_batch", "sov_lp_solve_family", "sov_batch_create", "sov_batch_solve", "sov_batch_results", "sov_batch_stats",
    "sov_batch_transfer_bytes", "sov_batch_destroy", "sov_autotune", "sov_spmv_csc", "sov_normal_factor_solve", "sov_normal_factor_solve_noalloc", "sov_device_info",
    "sov_last_error", "sov_mlp_create", "sov_mlp_param_count", "sov_mlp_get_params", "sov_mlp_set_params",
    "sov_mlp_forward", "sov_mlp_predict_start", "sov_mlp_loss_grad", "sov_mlp_train", "sov_mlp_destroy",
    "sov_lp_solve_batch_predicted", "sov_verify_solution", "sov_model_from_json", "sov_json_model_view",
    "sov_json_model_problem_type", "sov_json_model_variable_type", "sov_json_model_variable_name",
    "sov_json_model_row_name", "sov_json_model_destroy", "sov_presolve_lp", "sov_presolve_reduced",
    "sov_presolve_info", "sov_postsolve_lp", "sov_presolve_destroy", "sov_lp_solve_presolved",
]

_lib = None


class SovError(RuntimeError):
    pass


def load(build_if_missing: bool = True):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise SovError(f"{LIB_PATH} is missing; build it with python -m sovereign_b200.build")
        from .build import build
        build()
    lib = C.CDLL(LIB_PATH)
    M, O, R = C.POINTER(abi.SovModel), C.POINTER(abi.SovOptions), C.POINTER(abi.SovResult)
    lib.sov_default_lp_options.argtypes = [O]
    lib.sov_default_lp_options.restype = None
    lib.sov_default_qp_options.argtypes = [O]
    lib.sov_default_qp_options.restype = None
    lib.sov_ipm_dims.argtypes = [M, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
    lib.sov_lp_solve.argtypes = [M, O, R]
    lib.sov_qp_solve.argtypes = [M, O, R]
    lib.sov_lp_solve_batch.argtypes = [C.c_int32, M, O, C.c_int32, R]
    lib.sov_lp_solve_family.argtypes = [C.c_int32, M, O, C.c_int32, R]
    lib.sov_batch_create.argtypes = [C.c_int32, M, O, C.c_int32, C.POINTER(C.c_void_p)]
    lib.sov_batch_solve.argtypes = [C.c_void_p, C.c_void_p]
    lib.sov_batch_results.argtypes = [C.c_void_p, R]
    lib.sov_batch_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.sov_batch_transfer_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.sov_batch_destroy.argtypes = [C.c_void_p]
    lib.sov_batch_destroy.restype = None
    lib.sov_autotune.argtypes = [C.c_int32, M, O, C.c_char_p, C.c_char_p, C.c_int32]
    lib.sov_spmv_csc.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_int32]
    lib.sov_normal_factor_solve.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_int32, C.c_int32, C.c_void_p, C.c_int32, C.POINTER(C.c_int32)]
    lib.sov_normal_factor_solve_noalloc.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_int32),
                                                    C.c_void_p]
    lib.sov_device_info.argtypes = [C.c_char_p, C.c_int32]
    lib.sov_mlp_create.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(C.c_void_p)]
    lib.sov_mlp_param_count.argtypes = [C.c_void_p]
    lib.sov_mlp_param_count.restype = C.c_int64
    lib.sov_mlp_get_params.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    lib.sov_mlp_set_params.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    lib.sov_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p]
    lib.sov_mlp_predict_start.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_void_p, C.c_void_p,
                                          C.c_void_p]
    lib.sov_lp_solve_batch_predicted.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_int32,
                                                 C.c_void_p, C.c_void_p, C.c_void_p]
    lib.sov_mlp_loss_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.POINTER(C.c_double), C.c_void_p]
    lib.sov_mlp_train.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_float,
                                  C.c_uint64, C.POINTER(C.c_double)]
    lib.sov_mlp_destroy.argtypes = [C.c_void_p]
    lib.sov_mlp_destroy.restype = None
    lib.sov_verify_solution.argtypes = [M, R, C.c_double, C.POINTER(abi.SovCertificate)]
    lib.sov_model_from_json.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(C.c_void_p)]
    lib.sov_json_model_view.argtypes = [C.c_void_p]
    lib.sov_json_model_view.restype = M
    lib.sov_json_model_problem_type.argtypes = [C.c_void_p]
    lib.sov_json_model_variable_type.argtypes = [C.c_void_p, C.c_int32]
    lib.sov_json_model_variable_name.argtypes = [C.c_void_p, C.c_int32]
    lib.sov_json_model_variable_name.restype = C.c_char_p
    lib.sov_json_model_row_name.argtypes = [C.c_void_p, C.c_int32]
    lib.sov_json_model_row_name.restype = C.c_char_p
    lib.sov_json_model_destroy.argtypes = [C.c_void_p]
    lib.sov_json_model_destroy.restype = None
    lib.sov_presolve_lp.argtypes = [M, C.POINTER(C.c_void_p)]
    lib.sov_presolve_reduced.argtypes = [C.c_void_p]
    lib.sov_presolve_reduced.restype = M
    lib.sov_presolve_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int32)] * 4 + [C.c_char_p, C.c_int32]
    lib.sov_postsolve_lp.argtypes = [C.c_void_p, R, R]
    lib.sov_presolve_destroy.argtypes = [C.c_void_p]
    lib.sov_presolve_destroy.restype = None
    lib.sov_lp_solve_presolved.argtypes = [M, O, R]
    lib.sov_last_error.restype = C.c_char_p
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != 0:
        raise SovError(f"libsovipm error {rc}: {load().sov_last_error().decode(errors='replace')}")


def device_info() -> str:
    buf = C.create_string_buffer(256)
    check(load().sov_device_info(buf, 256))
    return buf.value.decode()
