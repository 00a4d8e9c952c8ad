"""ctypes mirror of include/sov_ipm.h (structs and enums only; no library is loaded here).

The same structures cross both the product library (``libsovipm.so``) and the test-only oracle
libraries, so a model is marshalled once and handed to either.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

# sovereign::SolverStatus (solver/core/include/sovereign/types.hpp:20-30)
OPTIMAL, FEASIBLE, INFEASIBLE, UNBOUNDED, TIME_LIMIT, ITERATION_LIMIT, NUMERICAL_ERROR, ERROR, \
    NOT_IMPLEMENTED = range(9)
STATUS_NAMES = ["OPTIMAL", "FEASIBLE", "INFEASIBLE", "UNBOUNDED", "TIME_LIMIT", "ITERATION_LIMIT",
                "NUMERICAL_ERROR", "ERROR", "NOT_IMPLEMENTED"]
# sovereign::ConstraintSense (types.hpp:12)
LE, GE, EQ = 0, 1, 2
PRECISION_FP64, PRECISION_MIXED = 0, 1
FACTOR_AUTO, FACTOR_DENSE, FACTOR_BANDED, FACTOR_XSPACE, FACTOR_SPARSE = 0, 1, 2, 3, 4
HISTORY_MAX = 128

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class SovModel(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("m", C.c_int32), ("maximize", C.c_int32), ("reserved", C.c_int32),
        ("col_ptr", _ip), ("row_idx", _ip), ("values", _dp), ("obj", _dp),
        ("obj_constant", C.c_double), ("lb", _dp), ("ub", _dp),
        ("sense", C.POINTER(C.c_int8)), ("rhs", _dp),
        ("q_col_ptr", _ip), ("q_row_idx", _ip), ("q_values", _dp),
    ]


class SovOptions(C.Structure):
    _fields_ = [
        ("max_iterations", C.c_int32), ("enable_scaling", C.c_int32),
        ("feasibility_tol", C.c_double), ("optimality_tol", C.c_double),
        ("fraction_to_boundary", C.c_double),
        ("precision", C.c_int32), ("factorization", C.c_int32),
        ("warm_x", _dp), ("warm_y", _dp), ("warm_s", _dp),
        ("pcg_max_iterations", C.c_int32), ("ipm_iterate_at", C.c_int32),
    ]


class SovDiagnostics(C.Structure):
    _fields_ = [
        ("scaling_applied", C.c_int32), ("history_len", C.c_int32),
        ("step_history_len", C.c_int32), ("refactorizations", C.c_int32),
        ("coefficient_min_abs_before", C.c_double), ("coefficient_max_abs_before", C.c_double),
        ("coefficient_min_abs_after", C.c_double), ("coefficient_max_abs_after", C.c_double),
        ("stall_iteration", C.c_int64),
        ("stall_gap", C.c_double), ("stall_mu", C.c_double),
        ("stall_primal_step", C.c_double), ("stall_dual_step", C.c_double),
        ("history_iterations", C.c_int64 * HISTORY_MAX),
        ("objective_history", C.c_double * HISTORY_MAX),
        ("gap_history", C.c_double * HISTORY_MAX),
        ("mu_history", C.c_double * HISTORY_MAX),
        ("primal_step_history", C.c_double * HISTORY_MAX),
        ("dual_step_history", C.c_double * HISTORY_MAX),
        ("fp64_fallbacks", C.c_int32), ("pcg_iterations", C.c_int32),
        ("warm_start_used", C.c_int32), ("structured_qp", C.c_int32),
    ]


class SovResult(C.Structure):
    _fields_ = [
        ("status", C.c_int32), ("iterations", C.c_int32), ("has_objective_value", C.c_int32),
        ("n_ipm", C.c_int32), ("m_ipm", C.c_int32),
        ("objective_value", C.c_double), ("duality_gap", C.c_double),
        ("primal_residual", C.c_double), ("dual_residual", C.c_double),
        ("primal", _dp), ("dual_col", _dp), ("dual_row", _dp),
        ("ipm_x", _dp), ("ipm_y", _dp), ("ipm_s", _dp),
        ("diagnostics", C.POINTER(SovDiagnostics)),
        ("solve_seconds", C.c_double),
        ("message", C.c_char * 512),
    ]


class SovCertificate(C.Structure):
    _fields_ = [
        ("is_valid", C.c_int32), ("issues", C.c_int32), ("nonfinite", C.c_int32), ("reserved", C.c_int32),
        ("max_bound_violation", C.c_double), ("max_constraint_violation", C.c_double),
        ("recomputed_objective", C.c_double), ("dual_objective", C.c_double),
        ("max_dual_infeasibility", C.c_double), ("relative_gap", C.c_double),
    ]


CERT_ISSUES = {1: "no feasible status", 2: "uncheckable status", 4: "non-finite", 8: "bound", 16: "constraint",
               32: "objective", 64: "gap"}


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_ip)


def default_options(qp: bool = False, precision: int = PRECISION_FP64,
                    factorization: int = FACTOR_AUTO, max_iterations: int | None = None) -> SovOptions:
    """InteriorPointOptions (interior_point.hpp:7-24) / QpInteriorPointOptions
    (qp_interior_point.hpp:7-18) defaults."""
    o = SovOptions()
    if qp:
        o.max_iterations, o.enable_scaling = 100, 0
        o.feasibility_tol = o.optimality_tol = 1e-8
    else:
        o.max_iterations, o.enable_scaling = 250, 1
        o.feasibility_tol = o.optimality_tol = 1e-9
    if max_iterations is not None:
        o.max_iterations = max_iterations
    o.fraction_to_boundary = 0.999
    o.precision = precision
    o.factorization = factorization
    o.pcg_max_iterations = 50
    return o
