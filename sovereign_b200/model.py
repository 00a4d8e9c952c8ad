"""Index-form LP/QP model (the arrays behind ``sov_model``) and its result.

``Model`` holds what a ``sovereign::OptimizationModel`` (solver/core/include/sovereign/types.hpp:
53-59) holds, with variable j named by its index and row i by its index: a CSC constraint matrix,
row senses and right-hand sides, column bounds, the linear objective and, for a QP, the stored
quadratic terms.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi


@dataclass
class Model:
    n: int
    m: int
    col_ptr: np.ndarray            # int32 n+1
    row_idx: np.ndarray            # int32 nnz
    values: np.ndarray             # float64 nnz
    obj: np.ndarray                # float64 n
    rhs: np.ndarray                # float64 m
    sense: np.ndarray              # int8 m
    lb: np.ndarray                 # float64 n
    ub: np.ndarray                 # float64 n
    obj_constant: float = 0.0
    maximize: bool = False
    q_col_ptr: np.ndarray | None = None
    q_row_idx: np.ndarray | None = None
    q_values: np.ndarray | None = None
    name: str = ""
    _keep: list = field(default_factory=list, repr=False)

    @property
    def nnz(self) -> int:
        return int(self.col_ptr[-1])

    @property
    def is_qp(self) -> bool:
        return self.q_col_ptr is not None

    def to_abi(self) -> abi.SovModel:
        """ctypes view; the arrays stay owned by this Model."""
        for a, dt in ((self.col_ptr, np.int32), (self.row_idx, np.int32), (self.values, np.float64),
                      (self.obj, np.float64), (self.rhs, np.float64), (self.lb, np.float64),
                      (self.ub, np.float64)):
            assert a.dtype == dt and a.flags["C_CONTIGUOUS"], a.dtype
        assert self.sense.dtype == np.int8
        s = abi.SovModel()
        s.n, s.m, s.maximize = self.n, self.m, int(self.maximize)
        s.col_ptr, s.row_idx, s.values = abi.iptr(self.col_ptr), abi.iptr(self.row_idx), abi.dptr(self.values)
        s.obj, s.obj_constant = abi.dptr(self.obj), float(self.obj_constant)
        s.lb, s.ub = abi.dptr(self.lb), abi.dptr(self.ub)
        s.sense = self.sense.ctypes.data_as(C.POINTER(C.c_int8))
        s.rhs = abi.dptr(self.rhs)
        if self.is_qp:
            s.q_col_ptr, s.q_row_idx, s.q_values = (abi.iptr(self.q_col_ptr), abi.iptr(self.q_row_idx),
                                                    abi.dptr(self.q_values))
        return s

    def dense_A(self) -> np.ndarray:
        A = np.zeros((self.m, self.n))
        for j in range(self.n):
            for k in range(self.col_ptr[j], self.col_ptr[j + 1]):
                A[self.row_idx[k], j] += self.values[k]
        return A

    def objective(self, x: np.ndarray) -> float:
        """Objective of the original model at x (constant included)."""
        v = float(self.obj_constant + self.obj @ x)
        if self.is_qp:
            for j in range(self.n):
                for k in range(self.q_col_ptr[j], self.q_col_ptr[j + 1]):
                    v += 0.5 * self.q_values[k] * x[self.q_row_idx[k]] * x[j]
        return v


def csc_from_columns(n: int, cols: list[list[tuple[int, float]]]):
    col_ptr = np.zeros(n + 1, dtype=np.int32)
    for j, c in enumerate(cols):
        col_ptr[j + 1] = col_ptr[j] + len(c)
    row_idx = np.fromiter((r for c in cols for r, _ in c), dtype=np.int32, count=int(col_ptr[-1]))
    values = np.fromiter((v for c in cols for _, v in c), dtype=np.float64, count=int(col_ptr[-1]))
    return col_ptr, row_idx, values


@dataclass
class Result:
    """Index-form sovereign::SolverResult (types.hpp:117-155)."""
    status: int
    iterations: int
    has_objective_value: bool
    objective_value: float
    duality_gap: float
    primal_residual: float
    dual_residual: float
    message: str
    primal: np.ndarray | None = None
    dual_col: np.ndarray | None = None
    dual_row: np.ndarray | None = None
    ipm_x: np.ndarray | None = None
    ipm_y: np.ndarray | None = None
    ipm_s: np.ndarray | None = None
    n_ipm: int = 0
    m_ipm: int = 0
    solve_seconds: float = 0.0
    diagnostics: dict | None = None

    @property
    def status_name(self) -> str:
        return abi.STATUS_NAMES[self.status]

    def dual(self) -> dict:
        """Name-keyed duals as the reference publishes them (interior_point.cpp:548,560)."""
        d = {}
        if self.dual_col is not None:
            d.update({f"x{j}": float(v) for j, v in enumerate(self.dual_col)})
        if self.dual_row is not None:
            d.update({f"row_{i}": float(v) for i, v in enumerate(self.dual_row)})
        return d


class ResultBuffers:
    """Caller-allocated output arrays for one sov_result."""

    def __init__(self, model: Model, with_ipm: bool = False, with_diag: bool = False,
                 n_ipm: int = 0, m_ipm: int = 0):
        self.primal = np.zeros(model.n)
        self.dual_col = np.zeros(model.n)
        self.dual_row = np.zeros(model.m)
        self.ipm = (np.zeros(n_ipm), np.zeros(m_ipm), np.zeros(n_ipm)) if with_ipm else None
        self.diag = abi.SovDiagnostics() if with_diag else None
        self.raw = abi.SovResult()
        r = self.raw
        r.primal, r.dual_col, r.dual_row = abi.dptr(self.primal), abi.dptr(self.dual_col), abi.dptr(self.dual_row)
        if self.ipm is not None:
            r.ipm_x, r.ipm_y, r.ipm_s = (abi.dptr(a) for a in self.ipm)
        if self.diag is not None:
            r.diagnostics = C.pointer(self.diag)

    def to_result(self) -> Result:
        r = self.raw
        diag = None
        if self.diag is not None:
            g = self.diag
            h, sh = g.history_len, g.step_history_len
            diag = dict(scaling_applied=bool(g.scaling_applied), refactorizations=g.refactorizations,
                        coefficient_min_abs_before=g.coefficient_min_abs_before,
                        coefficient_max_abs_before=g.coefficient_max_abs_before,
                        coefficient_min_abs_after=g.coefficient_min_abs_after,
                        coefficient_max_abs_after=g.coefficient_max_abs_after,
                        history_iterations=list(g.history_iterations[:h]),
                        objective_history=list(g.objective_history[:h]),
                        gap_history=list(g.gap_history[:h]), mu_history=list(g.mu_history[:h]),
                        primal_step_history=list(g.primal_step_history[:sh]),
                        dual_step_history=list(g.dual_step_history[:sh]),
                        stall_iteration=g.stall_iteration, fp64_fallbacks=g.fp64_fallbacks,
                        pcg_iterations=g.pcg_iterations, warm_start_used=bool(g.warm_start_used))
        res = Result(status=r.status, iterations=r.iterations, has_objective_value=bool(r.has_objective_value),
                     objective_value=r.objective_value, duality_gap=r.duality_gap,
                     primal_residual=r.primal_residual, dual_residual=r.dual_residual,
                     message=r.message.decode(errors="replace"), primal=self.primal.copy(),
                     dual_col=self.dual_col.copy(), dual_row=self.dual_row.copy(),
                     n_ipm=r.n_ipm, m_ipm=r.m_ipm, solve_seconds=r.solve_seconds, diagnostics=diag)
        if self.ipm is not None:
            res.ipm_x, res.ipm_y, res.ipm_s = (a.copy() for a in self.ipm)
        return res
