"""sov_normal_factor_solve_noalloc: the entry point for callers that cannot let the library allocate
device memory (they own all device memory and pass only their own buffers). Its answers must
equal the allocating entry point's, call after call, although every call reuses the same fixed
device array; sizes beyond its limit must be refused cleanly.

Collected last on purpose (file name), so a failure here does not hide the rest of the suite."""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from sovereign_b200 import _lib, problems as P
from sovereign_b200.ipm import normal_factor_solve

pytestmark = pytest.mark.gpu


def _device_call(torch, m, n, mdl, d, rhs):
    dev = torch.device("cuda:0")
    cp = torch.from_numpy(mdl.col_ptr).to(dev)
    ri = torch.from_numpy(mdl.row_idx).to(dev)
    va = torch.from_numpy(mdl.values).to(dev)
    dd = torch.from_numpy(np.ascontiguousarray(d)).to(dev)
    rr = torch.from_numpy(np.asfortranarray(rhs).reshape(-1, order="F").copy()).to(dev)
    nrhs = 1 if rhs.ndim == 1 else rhs.shape[1]
    dropped = C.c_int32(-1)
    stream = torch.cuda.current_stream().cuda_stream
    rc = _lib.load().sov_normal_factor_solve_noalloc(m, n, cp.data_ptr(), ri.data_ptr(), va.data_ptr(), dd.data_ptr(),
                                                     rr.data_ptr(), nrhs, C.byref(dropped), C.c_void_p(stream))
    out = rr.cpu().numpy().reshape((m, nrhs), order="F")
    return rc, (out[:, 0] if rhs.ndim == 1 else out), dropped.value


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    # second call: a transport system with one dependent row and weights large enough that both
    # entry points drop it (then the solution has no arbitrary component along the null vector)
    cases = [
        (P.random_sparse_lp(300, 1200, 4, 21), 8.0, 2, 1.0),  # IPM-like weights over 8 decades, 2 rhs
        (P.reference_transport(30), 0.6, 1, 100.0),          # a dependent row, a smaller system
    ]
    for mdl, spread, nrhs, scale in cases:
        m, n = mdl.m, mdl.n
        rng = np.random.default_rng(m)
        d = scale * 10.0 ** rng.uniform(-spread / 2, spread / 2, n)
        rhs = mdl.dense_A() @ rng.standard_normal((n, nrhs))
        rhs = rhs[:, 0] if nrhs == 1 else rhs
        want, want_drop = normal_factor_solve(m, n, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs)
        rc, got, got_drop = _device_call(torch, m, n, mdl, d, rhs)
        assert rc == 0
        assert got_drop == want_drop
        # same tolerance as the allocating path's own parity test against the oracle
        np.testing.assert_allclose(got, want, rtol=1e-7, atol=1e-9 * np.abs(want).max())


def test_noalloc_rejects_sizes_beyond_its_array():
    torch = pytest.importorskip("torch")
    mdl = P.random_sparse_lp(513, 600, 3, 5)
    d = np.ones(mdl.n)
    rhs = np.ones(mdl.m)
    rc, _, _ = _device_call(torch, mdl.m, mdl.n, mdl, d, rhs)
    assert rc == -4  # SOV_E_TOO_LARGE


def test_noalloc_refuses_bad_device_indices_without_writing():
    # the device arrays are never seen by the host: a row index outside [0, m) must be skipped on the
    # device and reported as SOV_E_ARGUMENT, and the next call must work as before
    torch = pytest.importorskip("torch")
    mdl = P.random_sparse_lp(40, 120, 3, 9)
    d = np.ones(mdl.n)
    rhs = np.ones(mdl.m)
    bad = mdl.row_idx.copy()
    bad[7] = mdl.m + 1000
    bad[11] = -3
    broken = dataclasses.replace(mdl, row_idx=bad)
    rc, _, _ = _device_call(torch, mdl.m, mdl.n, broken, d, rhs)
    assert rc == -1  # SOV_E_ARGUMENT
    assert b"row outside" in _lib.load().sov_last_error()
    want, _ = normal_factor_solve(mdl.m, mdl.n, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs)
    rc, got, _ = _device_call(torch, mdl.m, mdl.n, mdl, d, rhs)
    assert rc == 0
    np.testing.assert_allclose(got, want, rtol=1e-7, atol=1e-9 * np.abs(want).max())
