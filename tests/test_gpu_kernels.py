"""GPU kernel parity through the C ABI: SpMV bit-exact against the oracle (the reference's CPU
loop order), normal-equation factor/solve against the oracle's dense LU."""
import numpy as np
import pytest

import oracle
from sovereign_b200 import abi, problems as P
from sovereign_b200.ipm import normal_factor_solve, spmv_csc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("shape", [(90, 130, 5), (1, 1, 1), (2000, 10000, 8), (7, 300, 3)])
def test_spmv_bit_exact(shape):
    m, n, k = shape
    mdl = P.random_sparse_lp(m, n, min(k, m), 42)
    rng = np.random.default_rng(5)
    x = rng.standard_normal(n)
    x[::7] = 0.0
    y = rng.standard_normal(m)
    csc = (m, n, mdl.col_ptr, mdl.row_idx, mdl.values)
    assert np.array_equal(spmv_csc(m, n, mdl.col_ptr, mdl.row_idx, mdl.values, x), oracle.spmv(csc, x))
    assert np.array_equal(spmv_csc(m, n, mdl.col_ptr, mdl.row_idx, mdl.values, y, transpose=True),
                          oracle.spmv(csc, y, transpose=True))


def test_spmv_empty_columns():
    mdl = P.bounded_lp_example()
    x = np.array([1.0, 2.0, 3.0])
    assert np.array_equal(spmv_csc(3, 3, mdl.col_ptr, mdl.row_idx, mdl.values, x),
                          oracle.spmv((3, 3, mdl.col_ptr, mdl.row_idx, mdl.values), x))


@pytest.mark.parametrize("m,n,spread", [(60, 150, 6), (200, 1000, 10), (513, 2000, 4)])
def test_normal_factor_solve_fp64(m, n, spread):
    mdl = P.random_sparse_lp(m, n, 4, 12345)
    rng = np.random.default_rng(m)
    d = 10.0 ** rng.uniform(-spread / 2, spread / 2, n)  # IPM diagonals spanning 10^spread
    rhs = rng.standard_normal((m, 2))
    z, dropped = normal_factor_solve(m, n, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs)
    rc, zo = oracle.normal_factor_solve(m, n, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs)
    assert rc == 0 and dropped == 0
    np.testing.assert_allclose(z, zo, rtol=1e-7, atol=1e-9 * np.abs(zo).max())


def test_normal_factor_solve_fp32_is_a_preconditioner_grade_solve():
    mdl = P.random_sparse_lp(300, 1200, 4, 3)
    d = np.random.default_rng(0).uniform(0.5, 2.0, 1200)
    rhs = np.random.default_rng(1).standard_normal(300)
    z, _ = normal_factor_solve(300, 1200, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs,
                               precision=abi.PRECISION_MIXED)
    _, zo = oracle.normal_factor_solve(300, 1200, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs)
    assert np.linalg.norm(z - zo) / np.linalg.norm(zo) < 1e-4


def test_banded_equals_dense():
    mdl = P.convex_sequence_qp(600, 1)
    d = np.random.default_rng(0).uniform(0.1, 10.0, mdl.n)
    rhs = np.random.default_rng(1).standard_normal(mdl.m)
    zb, _ = normal_factor_solve(mdl.m, mdl.n, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs,
                                factorization=abi.FACTOR_BANDED)
    zd, _ = normal_factor_solve(mdl.m, mdl.n, mdl.col_ptr, mdl.row_idx, mdl.values, d, rhs,
                                factorization=abi.FACTOR_DENSE)
    np.testing.assert_allclose(zb, zd, rtol=1e-7, atol=1e-9 * np.abs(zd).max())
