"""Python face of the engine, shaped like the reference's solver classes.

``InteriorPointSolver(InteriorPointOptions).solve(model)`` mirrors
sovereign::InteriorPointSolver (solver/lp/include/sovereign/interior_point.hpp:26-36) and
``QpInteriorPointSolver`` mirrors solver/qp/include/sovereign/qp_interior_point.hpp:21-31: same
option names and defaults, same statuses and messages, results with the same fields
(``objective_value``, ``primal``, ``dual``, ``duality_gap``, residuals, ``iterations``). Every
call goes through the C ABI of libsovipm.so; there is no Python or CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import abi
from ._lib import check, load
from .model import Model, Result, ResultBuffers


@dataclass
class InteriorPointOptions:
    """InteriorPointOptions (interior_point.hpp:7-24) plus the engine's precision knob."""
    max_iterations: int = 250
    feasibility_tol: float = 1e-9
    optimality_tol: float = 1e-9
    fraction_to_boundary: float = 0.999
    enable_scaling: bool = True
    use_sparse_normal_equations: bool = False
    precision: int = abi.PRECISION_FP64
    pcg_max_iterations: int = 50
    ipm_iterate_at: int = 0   # iterate returned in ipm_x/y/s: 0 final, k >= 1 start of iteration k

    def to_abi(self, qp: bool = False) -> abi.SovOptions:
        o = abi.default_options(qp=qp)
        o.max_iterations = self.max_iterations
        o.feasibility_tol = self.feasibility_tol
        o.optimality_tol = self.optimality_tol
        o.fraction_to_boundary = self.fraction_to_boundary
        o.enable_scaling = int(self.enable_scaling) if not qp else 0
        o.precision = self.precision
        o.pcg_max_iterations = self.pcg_max_iterations
        o.ipm_iterate_at = self.ipm_iterate_at
        if qp:
            # SOVEREIGN_QP_KKT (qp_interior_point.cpp:418-422): "sparse" takes the quasi-definite KKT
            # system, "dense" a dense factorization of the engine's system
            mode = os.environ.get("SOVEREIGN_QP_KKT", "auto")
        else:
            mode = os.environ.get("SOVEREIGN_IPM_NORMAL_EQUATIONS", "auto")  # interior_point.cpp:132-133
        o.factorization = {"dense": abi.FACTOR_DENSE, "banded": abi.FACTOR_BANDED,
                           "sparse": abi.FACTOR_SPARSE}.get(mode, abi.FACTOR_AUTO)
        return o


@dataclass
class QpInteriorPointOptions(InteriorPointOptions):
    """QpInteriorPointOptions (qp_interior_point.hpp:7-18)."""
    max_iterations: int = 100
    feasibility_tol: float = 1e-8
    optimality_tol: float = 1e-8
    enable_scaling: bool = False


def _dims(model: Model) -> tuple[int, int]:
    n = C.c_int32()
    m = C.c_int32()
    check(load().sov_ipm_dims(C.byref(model.to_abi()), int(model.is_qp), C.byref(n), C.byref(m)))
    return n.value, m.value


def _solve(model: Model, opt: abi.SovOptions, qp: bool, with_ipm: bool, with_diag: bool,
           warm: tuple | None) -> Result:
    n_ipm, m_ipm = _dims(model)
    buf = ResultBuffers(model, with_ipm=with_ipm, with_diag=with_diag, n_ipm=n_ipm, m_ipm=m_ipm)
    keep = None
    if warm is not None:
        keep = [np.ascontiguousarray(a, dtype=np.float64) for a in warm]
        opt.warm_x, opt.warm_y, opt.warm_s = (abi.dptr(a) for a in keep)
    sm = model.to_abi()
    fn = load().sov_qp_solve if qp else load().sov_lp_solve
    check(fn(C.byref(sm), C.byref(opt), C.byref(buf.raw)))
    del keep
    return buf.to_result()


class InteriorPointSolver:
    """Mehrotra predictor-corrector LP interior point on the B200 (drop-in for
    sovereign::InteriorPointSolver)."""

    def __init__(self, options: InteriorPointOptions | None = None):
        self.options = options or InteriorPointOptions()

    def solve(self, model: Model, with_ipm: bool = False, with_diag: bool = False,
              warm_start: tuple | None = None) -> Result:
        return _solve(model, self.options.to_abi(qp=False), False, with_ipm, with_diag, warm_start)


class QpInteriorPointSolver:
    """Convex-QP interior point on the B200: y-space normal equations for separable Hessians, a
    dense H or the sparse quasi-definite KKT system for Hessians that couple variables."""

    def __init__(self, options: QpInteriorPointOptions | None = None):
        self.options = options or QpInteriorPointOptions()

    def solve(self, model: Model, with_ipm: bool = False, with_diag: bool = False) -> Result:
        return _solve(model, self.options.to_abi(qp=True), True, with_ipm, with_diag, None)


def _per_lp_options(opt: abi.SovOptions, warm_starts: list):
    """One option block per LP (copies of opt) carrying each LP's warm start, if any; the arrays
    the blocks point at are returned too and must outlive the call."""
    keep = []
    opts = (abi.SovOptions * len(warm_starts))()
    for k, w in enumerate(warm_starts):
        C.memmove(C.byref(opts[k]), C.byref(opt), C.sizeof(abi.SovOptions))
        if w is not None:
            a = [np.ascontiguousarray(v, dtype=np.float64) for v in w]
            keep.append(a)
            opts[k].warm_x, opts[k].warm_y, opts[k].warm_s = (abi.dptr(v) for v in a)
    return opts, keep


def _struct_dtype(T) -> np.dtype:
    """numpy view of a ctypes structure of the ABI, pointers as uint64 addresses."""
    names, formats, offsets = [], [], []
    for name, ctype in T._fields_:
        names.append(name)
        offsets.append(getattr(T, name).offset)
        if isinstance(ctype, type) and issubclass(ctype, (C._Pointer, C.c_void_p)):
            formats.append(np.uint64)
        else:
            formats.append(np.dtype(ctype))
    return np.dtype(dict(names=names, formats=formats, offsets=offsets, itemsize=C.sizeof(T)))


_MODEL_DT = None
_RESULT_DT = None


def _addr(a: np.ndarray) -> int:
    return a.__array_interface__["data"][0]


def _addrs(arrs: list) -> list[int]:
    """Data addresses of many arrays: through a ctypes view where the array is writable (about a
    third of the cost of building __array_interface__), else through the interface."""
    out = []
    for a in arrs:
        try:
            out.append(C.addressof(C.c_char.from_buffer(a)) if a.size else _addr(a))
        except (TypeError, ValueError, BufferError):
            out.append(_addr(a))
    return out


def _marshal(models: list[Model], with_ipm: bool):
    """The models as one array of sov_model and one array of sov_result whose outputs are views
    of one float64 buffer, built column-wise: no per-LP ctypes objects."""
    global _MODEL_DT, _RESULT_DT
    if _MODEL_DT is None:
        _MODEL_DT, _RESULT_DT = _struct_dtype(abi.SovModel), _struct_dtype(abi.SovResult)
    k = len(models)
    M = np.zeros(k, dtype=_MODEL_DT)
    for name, key in (("col_ptr", "col_ptr"), ("row_idx", "row_idx"), ("values", "values"), ("obj", "obj"),
                      ("lb", "lb"), ("ub", "ub"), ("sense", "sense"), ("rhs", "rhs")):
        arrs = [getattr(m, key) for m in models]
        want = np.int8 if key == "sense" else np.int32 if key in ("col_ptr", "row_idx") else np.float64
        for a in arrs:
            if a.dtype != want or not a.flags.c_contiguous:
                raise TypeError(f"Model.{key} must be a contiguous {np.dtype(want)} array")
        M[name] = _addrs(arrs)
    M["n"] = [m.n for m in models]
    M["m"] = [m.m for m in models]
    M["maximize"] = [int(m.maximize) for m in models]
    M["obj_constant"] = [float(m.obj_constant) for m in models]
    n = M["n"].astype(np.int64)
    mm = M["m"].astype(np.int64)
    dims = [_dims(m) for m in models] if with_ipm else None
    ni = np.array([d[0] for d in dims], dtype=np.int64) if with_ipm else np.zeros(k, np.int64)
    mi = np.array([d[1] for d in dims], dtype=np.int64) if with_ipm else np.zeros(k, np.int64)
    sizes = 2 * n + mm + 2 * ni + mi
    start = np.concatenate([[0], np.cumsum(sizes)])
    buf = np.zeros(int(start[-1]) if k else 0)
    base = _addr(buf) if buf.size else 0
    R = np.zeros(k, dtype=_RESULT_DT)
    off = start[:-1]
    R["primal"] = base + 8 * off
    R["dual_col"] = base + 8 * (off + n)
    R["dual_row"] = base + 8 * (off + 2 * n)
    if with_ipm:
        R["ipm_x"] = base + 8 * (off + 2 * n + mm)
        R["ipm_y"] = base + 8 * (off + 2 * n + mm + ni)
        R["ipm_s"] = base + 8 * (off + 2 * n + mm + ni + mi)
    return M, R, buf, (off, n, mm, ni, mi)


def _unmarshal(R: np.ndarray, buf: np.ndarray, layout, with_ipm: bool) -> list[Result]:
    off, n, mm, ni, mi = layout
    k = len(R)
    # the record fields as Python lists in one pass each (per-LP numpy scalar access costs more)
    status, its, has = R["status"].tolist(), R["iterations"].tolist(), R["has_objective_value"].tolist()
    obj, gap = R["objective_value"].tolist(), R["duality_gap"].tolist()
    pres, dres = R["primal_residual"].tolist(), R["dual_residual"].tolist()
    nip, mip, secs = R["n_ipm"].tolist(), R["m_ipm"].tolist(), R["solve_seconds"].tolist()
    width = R.dtype["message"].itemsize  # the whole char array of a record
    msgs = np.ascontiguousarray(R["message"]).view(f"S{width}").reshape(k).tolist() if k else []
    offl, nl, ml = off.tolist(), n.tolist(), mm.tolist()
    nil, mil = (ni.tolist(), mi.tolist()) if with_ipm else (None, None)
    out = []
    for q in range(k):
        o, a, b = offl[q], nl[q], ml[q]
        r = Result(status=status[q], iterations=its[q], has_objective_value=bool(has[q]),
                   objective_value=obj[q], duality_gap=gap[q], primal_residual=pres[q],
                   dual_residual=dres[q], message=msgs[q].split(b"\0", 1)[0].decode(errors="replace"),
                   primal=buf[o:o + a], dual_col=buf[o + a:o + 2 * a], dual_row=buf[o + 2 * a:o + 2 * a + b],
                   n_ipm=nip[q], m_ipm=mip[q], solve_seconds=secs[q])
        if with_ipm:
            p, x, y = o + 2 * a + b, nil[q], mil[q]
            r.ipm_x, r.ipm_y, r.ipm_s = buf[p:p + x], buf[p + x:p + x + y], buf[p + x + y:p + 2 * x + y]
        out.append(r)
    return out


def _solve_many(entry, models: list[Model], options, with_ipm: bool, warm_starts, with_diag: bool) -> list[Result]:
    """sov_lp_solve_batch / sov_lp_solve_family through the column-wise marshalling (results with
    diagnostics take the per-LP buffers)."""
    opt = (options or InteriorPointOptions()).to_abi()
    if with_diag or any(m.is_qp for m in models):
        return None
    M, R, buf, layout = _marshal(models, with_ipm)
    mp = C.cast(C.c_void_p(_addr(M)), C.POINTER(abi.SovModel)) if len(models) else None
    rp = C.cast(C.c_void_p(_addr(R)), C.POINTER(abi.SovResult)) if len(models) else None
    if warm_starts is None:
        check(entry(len(models), mp, C.byref(opt), 0, rp))
    else:
        opts, keep = _per_lp_options(opt, warm_starts)
        check(entry(len(models), mp, opts, C.sizeof(abi.SovOptions), rp))
        del keep
    return _unmarshal(R, buf, layout, with_ipm)


def solve_batch(models: list[Model], options: InteriorPointOptions | None = None, with_ipm: bool = False,
                warm_starts: list | None = None, with_diag: bool = False) -> list[Result]:
    """Independent LPs in one persistent batched launch (sov_lp_solve_batch). warm_starts: one
    (x, y, s) tuple (engine standard form) or None per LP; passed as per-LP option blocks."""
    fast = _solve_many(load().sov_lp_solve_batch, models, options, with_ipm, warm_starts, with_diag)
    if fast is not None:
        return fast
    opt = (options or InteriorPointOptions()).to_abi()
    bufs = []
    for m in models:
        n_ipm, m_ipm = _dims(m) if with_ipm else (0, 0)
        bufs.append(ResultBuffers(m, with_ipm=with_ipm, with_diag=with_diag, n_ipm=n_ipm, m_ipm=m_ipm))
    arr = (abi.SovModel * len(models))(*[m.to_abi() for m in models])
    res = (abi.SovResult * len(models))(*[b.raw for b in bufs])
    if warm_starts is None:
        check(load().sov_lp_solve_batch(len(models), arr, C.byref(opt), 0, res))
    else:
        opts, keep = _per_lp_options(opt, warm_starts)
        check(load().sov_lp_solve_batch(len(models), arr, opts, C.sizeof(abi.SovOptions), res))
        del keep
    out = []
    for b, r in zip(bufs, res):
        b.raw = r
        out.append(b.to_result())
    return out


def solve_family(models: list[Model], options: InteriorPointOptions | None = None, with_ipm: bool = False,
                 warm_starts: list | None = None, with_diag: bool = False) -> list[Result]:
    """LPs of one parametric family -- the same A, bounds and senses, their own b, c -- solved
    together (sov_lp_solve_family): one symbolic analysis, up to 64 LPs per launch with their
    vectors interleaved. Arguments as solve_batch."""
    fast = _solve_many(load().sov_lp_solve_family, models, options, with_ipm, warm_starts, with_diag)
    if fast is not None:
        return fast
    opt = (options or InteriorPointOptions()).to_abi()
    bufs = []
    for m in models:
        n_ipm, m_ipm = _dims(m) if with_ipm else (0, 0)
        bufs.append(ResultBuffers(m, with_ipm=with_ipm, with_diag=with_diag, n_ipm=n_ipm, m_ipm=m_ipm))
    arr = (abi.SovModel * len(models))(*[m.to_abi() for m in models])
    res = (abi.SovResult * len(models))(*[b.raw for b in bufs])
    if warm_starts is None:
        check(load().sov_lp_solve_family(len(models), arr, C.byref(opt), 0, res))
    else:
        opts, keep = _per_lp_options(opt, warm_starts)
        check(load().sov_lp_solve_family(len(models), arr, opts, C.sizeof(abi.SovOptions), res))
        del keep
    out = []
    for b, r in zip(bufs, res):
        b.raw = r
        out.append(b.to_result())
    return out


class DeviceBatch:
    """A prepared batch resident on the device (sov_batch_*): upload once, solve many times."""

    def __init__(self, models: list[Model], options: InteriorPointOptions | None = None,
                 warm_starts: list | None = None):
        self.models = models
        self._arr = (abi.SovModel * len(models))(*[m.to_abi() for m in models])
        self._opt = (options or InteriorPointOptions()).to_abi()
        h = C.c_void_p()
        if warm_starts is None:
            check(load().sov_batch_create(len(models), self._arr, C.byref(self._opt), 0, C.byref(h)))
        else:
            opts, keep = _per_lp_options(self._opt, warm_starts)
            check(load().sov_batch_create(len(models), self._arr, opts, C.sizeof(abi.SovOptions), C.byref(h)))
            del keep
        self.handle = h

    def solve(self, stream: int = 0) -> None:
        check(load().sov_batch_solve(self.handle, C.c_void_p(stream)))

    def results(self, with_ipm: bool = False) -> list[Result]:
        bufs = []
        for m in self.models:
            n_ipm, m_ipm = _dims(m) if with_ipm else (0, 0)
            bufs.append(ResultBuffers(m, with_ipm=with_ipm, n_ipm=n_ipm, m_ipm=m_ipm))
        res = (abi.SovResult * len(self.models))(*[b.raw for b in bufs])
        check(load().sov_batch_results(self.handle, res))
        out = []
        for b, r in zip(bufs, res):
            b.raw = r
            out.append(b.to_result())
        return out

    def stats(self) -> dict:
        launches = C.c_int32()
        ms, byts, flops = C.c_double(), C.c_double(), C.c_double()
        check(load().sov_batch_stats(self.handle, C.byref(launches), C.byref(ms), C.byref(byts), C.byref(flops)))
        return dict(launches=launches.value, kernel_ms=ms.value, bytes_per_iteration=byts.value,
                    flops_per_iteration=flops.value)

    def close(self) -> None:
        if self.handle:
            load().sov_batch_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def autotune(models: list[Model], options: InteriorPointOptions | None = None, tuning_file: str | None = None) -> str:
    arr = (abi.SovModel * len(models))(*[m.to_abi() for m in models])
    opt = (options or InteriorPointOptions()).to_abi()
    rep = C.create_string_buffer(4096)
    check(load().sov_autotune(len(models), arr, C.byref(opt), tuning_file.encode() if tuning_file else None, rep, 4096))
    return rep.value.decode()


def spmv_csc(m: int, n: int, col_ptr, row_idx, values, x, transpose: bool = False) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros(n if transpose else m)
    check(load().sov_spmv_csc(m, n, col_ptr.ctypes.data, row_idx.ctypes.data, values.ctypes.data, x.ctypes.data,
                              y.ctypes.data, int(transpose)))
    return y


def normal_factor_solve(m: int, n: int, col_ptr, row_idx, values, d, rhs, precision: int = abi.PRECISION_FP64,
                        factorization: int = abi.FACTOR_AUTO):
    d = np.ascontiguousarray(d, dtype=np.float64)
    rhs = np.array(rhs, dtype=np.float64, order="F", copy=True)
    nrhs = 1 if rhs.ndim == 1 else rhs.shape[1]
    dropped = C.c_int32()
    check(load().sov_normal_factor_solve(m, n, col_ptr.ctypes.data, row_idx.ctypes.data, values.ctypes.data,
                                         d.ctypes.data, precision, factorization, rhs.ctypes.data, nrhs,
                                         C.byref(dropped)))
    return rhs, dropped.value


def verify_solution(model: Model, result: Result, tol: float = 1e-6) -> dict:
    """Certificate of `result` against `model` on the GPU (sov_verify_solution): the checks of
    SolutionVerifier::verify (solver/core/src/verifier.cpp:10-150, default tolerance 1e-6) plus the
    dual side (reduced-cost and row-dual signs, dual objective, relative gap)."""
    r = abi.SovResult()
    primal = np.ascontiguousarray(result.primal, dtype=np.float64)
    dual_row = np.ascontiguousarray(result.dual_row, dtype=np.float64)
    r.primal, r.dual_row = abi.dptr(primal), abi.dptr(dual_row)
    r.status, r.has_objective_value = result.status, int(result.has_objective_value)
    r.objective_value, r.duality_gap = result.objective_value, result.duality_gap
    cert = abi.SovCertificate()
    check(load().sov_verify_solution(C.byref(model.to_abi()), C.byref(r), tol, C.byref(cert)))
    out = {k: getattr(cert, k) for k, _ in abi.SovCertificate._fields_ if k != "reserved"}
    out["is_valid"] = bool(cert.is_valid)
    out["issue_names"] = [v for k, v in abi.CERT_ISSUES.items() if cert.issues & k]
    return out


def load_model_json(text: str | bytes) -> tuple[Model, list[str], list[str]]:
    """A model in the reference's JSON format (solver/core/src/json_io.cpp:13-80), read by the
    CSC-native ingest (sov_model_from_json, host only): (Model, variable names, row names)."""
    data = text.encode() if isinstance(text, str) else bytes(text)
    h = C.c_void_p()
    lib = load()
    check(lib.sov_model_from_json(data, len(data), C.byref(h)))
    try:
        v = lib.sov_json_model_view(h).contents
        n, m = v.n, v.m
        nnz = v.col_ptr[n] if n > 0 else 0

        def arr(ptr, count, dtype):
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True) if count else np.zeros(0, dtype)

        mdl = Model(n=n, m=m, col_ptr=arr(v.col_ptr, n + 1, np.int32) if n else np.zeros(1, np.int32),
                    row_idx=arr(v.row_idx, nnz, np.int32), values=arr(v.values, nnz, np.float64),
                    obj=arr(v.obj, n, np.float64), rhs=arr(v.rhs, m, np.float64),
                    sense=np.array([v.sense[i] for i in range(m)], dtype=np.int8), lb=arr(v.lb, n, np.float64),
                    ub=arr(v.ub, n, np.float64), obj_constant=v.obj_constant, maximize=bool(v.maximize))
        if v.q_col_ptr:
            qn = v.q_col_ptr[n]
            mdl.q_col_ptr = arr(v.q_col_ptr, n + 1, np.int32)
            mdl.q_row_idx = arr(v.q_row_idx, qn, np.int32)
            mdl.q_values = arr(v.q_values, qn, np.float64)
        names = [lib.sov_json_model_variable_name(h, j).decode() for j in range(n)]
        rows = [lib.sov_json_model_row_name(h, i).decode() for i in range(m)]
    finally:
        lib.sov_json_model_destroy(h)
    return mdl, names, rows


class Presolved:
    """LP presolve in index form (sov_presolve_lp): `reduced` is the model to solve (when `status`
    is None; else presolve decided the status), `postsolve(result)` maps its answer back to the
    original columns and rows (sov_postsolve_lp). Host only."""

    def __init__(self, model: Model):
        self.model = model
        self._abi = model.to_abi()
        self.h = C.c_void_p()
        check(load().sov_presolve_lp(C.byref(self._abi), C.byref(self.h)))
        st, rr, cr, bt = (C.c_int32() for _ in range(4))
        msg = C.create_string_buffer(512)
        check(load().sov_presolve_info(self.h, C.byref(st), C.byref(rr), C.byref(cr), C.byref(bt), msg, 512))
        self.status = None if st.value < 0 else st.value
        self.rows_removed, self.cols_removed, self.bounds_tightened = rr.value, cr.value, bt.value
        self.message = msg.value.decode()
        v = load().sov_presolve_reduced(self.h).contents
        n, m = v.n, v.m
        nnz = v.col_ptr[n] if n > 0 else 0

        def arr(ptr, count, dtype):
            return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True) if count else np.zeros(0, dtype)

        self.reduced = Model(n=n, m=m, col_ptr=arr(v.col_ptr, n + 1, np.int32), row_idx=arr(v.row_idx, nnz, np.int32),
                             values=arr(v.values, nnz, np.float64), obj=arr(v.obj, n, np.float64),
                             rhs=arr(v.rhs, m, np.float64), sense=np.array([v.sense[i] for i in range(m)], np.int8),
                             lb=arr(v.lb, n, np.float64), ub=arr(v.ub, n, np.float64),
                             obj_constant=v.obj_constant, maximize=bool(v.maximize))

    def postsolve(self, reduced: Result | None) -> Result:
        full = ResultBuffers(self.model, with_diag=False)
        if reduced is None:
            check(load().sov_postsolve_lp(self.h, None, C.byref(full.raw)))
            return full.to_result()
        rb = ResultBuffers(self.reduced)
        r = rb.raw
        r.status, r.iterations, r.has_objective_value = reduced.status, reduced.iterations, int(reduced.has_objective_value)
        r.objective_value, r.duality_gap = reduced.objective_value, reduced.duality_gap
        r.primal_residual, r.dual_residual = reduced.primal_residual, reduced.dual_residual
        r.message = reduced.message.encode()[:511]
        rb.primal[:] = reduced.primal
        rb.dual_row[:] = reduced.dual_row
        if reduced.dual_col is not None:
            rb.dual_col[:] = reduced.dual_col
        check(load().sov_postsolve_lp(self.h, C.byref(r), C.byref(full.raw)))
        return full.to_result()

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            load().sov_presolve_destroy(self.h)
            self.h = C.c_void_p()


def solve_presolved(model: Model, options: InteriorPointOptions | None = None, with_diag: bool = False) -> Result:
    """Presolve, the GPU IPM on the reduced LP, postsolve (sov_lp_solve_presolved)."""
    opt = (options or InteriorPointOptions()).to_abi()
    buf = ResultBuffers(model, with_diag=with_diag)
    check(load().sov_lp_solve_presolved(C.byref(model.to_abi()), C.byref(opt), C.byref(buf.raw)))
    return buf.to_result()
