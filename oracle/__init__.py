"""TEST INFRASTRUCTURE ONLY -- the CPU oracle of the GPU interior-point engine.

* ``restatement``: libsovoracle.so, the plain-C restatement of the reference's IPM (ipm_oracle.c).
* ``reference``:   _ref/libsovref.so, the reference's own solvers compiled unmodified by
                   oracle/Makefile (only present where the reference sources were available at
                   build time; the built file travels with the repository snapshot).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py import this
package. The product (``sovereign_b200``) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from sovereign_b200 import abi
from sovereign_b200.model import Model, ResultBuffers

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_PATH = os.path.join(HERE, "libsovoracle.so")
REFERENCE_PATH = os.path.join(HERE, "_ref", "libsovref.so")
# the reference checkout: the one place its location is set (SOVEREIGN_REFERENCE_DIR overrides)
REFERENCE_DIR = os.environ.get("SOVEREIGN_REFERENCE_DIR", "/root/reference")
REFERENCE_SRC = os.path.join(REFERENCE_DIR, "solver", "lp", "src", "interior_point.cpp")


def build(reference: bool = True) -> None:
    """Compile the restatement, and the reference library when its sources are present."""
    target = ["all"] if reference and os.path.exists(REFERENCE_SRC) else ["oracle"]
    subprocess.run(["make", "-s", "-C", HERE, f"REF={REFERENCE_DIR}"] + target, check=True)


_libs: dict = {}


def _load(path: str, kind: str):
    if kind in _libs:
        return _libs[kind]
    if not os.path.exists(path):
        build(reference=(kind == "reference"))
    lib = C.CDLL(path)
    if kind == "restatement":
        lib.oracle_lp_solve.argtypes = [C.POINTER(abi.SovModel), C.POINTER(abi.SovOptions), C.POINTER(abi.SovResult)]
        lib.oracle_qp_solve.argtypes = lib.oracle_lp_solve.argtypes
        lib.oracle_spmv_csc.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_int32]
        lib.oracle_normal_factor_solve.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                                   C.c_void_p, C.c_void_p, C.c_int32]
        lib.oracle_ipm_form.argtypes = [C.POINTER(abi.SovModel), C.c_int32] + [C.c_void_p] * 3 + [C.c_int32] + \
            [C.c_void_p] * 5
    else:
        lib.ref_solve.argtypes = [C.POINTER(abi.SovModel), C.c_int32, C.c_int32, C.POINTER(abi.SovResult)]
        lib.ref_solve.restype = C.c_double
        lib.ref_solve_many.argtypes = [C.c_int32, C.POINTER(abi.SovModel), C.c_int32, C.c_void_p, C.c_void_p,
                                       C.c_void_p]
        lib.ref_solve_many.restype = C.c_double
        lib.ref_hardware_threads.restype = C.c_int32
    _libs[kind] = lib
    return lib


def restatement():
    return _load(RESTATEMENT_PATH, "restatement")


def reference():
    return _load(REFERENCE_PATH, "reference")


def reference_available() -> bool:
    return os.path.exists(REFERENCE_PATH) or os.path.exists(REFERENCE_SRC)


def _dims(model: Model, qp: bool) -> tuple[int, int]:
    n_ub = int(np.sum((model.ub < 1e29) & np.isfinite(model.ub)))
    n_slack = int(np.sum(model.sense != abi.EQ)) + n_ub
    return model.n + n_slack, model.m + n_ub


def solve(model: Model, qp: bool | None = None, kind: str = "restatement", max_iterations: int | None = None,
          with_ipm: bool = False, with_diag: bool = False, options: abi.SovOptions | None = None):
    """Solve through the restatement or the reference; returns sovereign_b200.model.Result."""
    qp = model.is_qp if qp is None else qp
    n_ipm, m_ipm = _dims(model, qp)
    buf = ResultBuffers(model, with_ipm=with_ipm and kind == "restatement", with_diag=with_diag,
                        n_ipm=n_ipm, m_ipm=m_ipm)
    sm = model.to_abi()
    if kind == "restatement":
        opt = options or abi.default_options(qp=qp, max_iterations=max_iterations)
        fn = restatement().oracle_qp_solve if qp else restatement().oracle_lp_solve
        fn(C.byref(sm), C.byref(opt), C.byref(buf.raw))
    else:
        reference().ref_solve(C.byref(sm), int(qp), int(max_iterations or 0), C.byref(buf.raw))
    return buf.to_result()


def solve_many_reference(models: list[Model], threads: int = 0):
    """Wall seconds for the reference to solve all models on `threads` host threads."""
    arr = (abi.SovModel * len(models))(*[m.to_abi() for m in models])
    obj = np.zeros(len(models))
    its = np.zeros(len(models), dtype=np.int32)
    st = np.zeros(len(models), dtype=np.int32)
    secs = reference().ref_solve_many(len(models), arr, threads, obj.ctypes.data, its.ctypes.data, st.ctypes.data)
    return secs, obj, its, st


def spmv(model_or_csc, x: np.ndarray, transpose: bool = False) -> np.ndarray:
    m, n, cp, ri, v = model_or_csc
    y = np.zeros(n if transpose else m)
    restatement().oracle_spmv_csc(m, n, cp.ctypes.data, ri.ctypes.data, v.ctypes.data, x.ctypes.data,
                                  y.ctypes.data, int(transpose))
    return y


def normal_factor_solve(m, n, cp, ri, v, d, rhs):
    rhs = np.array(rhs, dtype=np.float64, order="F")
    nrhs = 1 if rhs.ndim == 1 else rhs.shape[1]
    rc = restatement().oracle_normal_factor_solve(m, n, cp.ctypes.data, ri.ctypes.data, v.ctypes.data,
                                                  d.ctypes.data, rhs.ctypes.data, nrhs)
    return rc, rhs


def ipm_form(model: Model, enable_scaling: bool = True):
    n_ipm, m_ipm = _dims(model, False)
    cap = model.nnz + n_ipm + 8
    cp = np.zeros(n_ipm + 1, dtype=np.int32)
    ri = np.zeros(cap, dtype=np.int32)
    v = np.zeros(cap)
    b, c = np.zeros(m_ipm), np.zeros(n_ipm)
    cs, rs, sh = np.zeros(n_ipm), np.zeros(m_ipm), np.zeros(model.n)
    sm = model.to_abi()
    nnz = restatement().oracle_ipm_form(C.byref(sm), int(enable_scaling), cp.ctypes.data, ri.ctypes.data,
                                        v.ctypes.data, cap, b.ctypes.data, c.ctypes.data, cs.ctypes.data,
                                        rs.ctypes.data, sh.ctypes.data)
    return dict(col_ptr=cp, row_idx=ri[:nnz], values=v[:nnz], b=b, c=c, col_scale=cs, row_scale=rs, shift=sh,
                m=m_ipm, n=n_ipm)
