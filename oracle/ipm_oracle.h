/* ipm_oracle.h -- TEST INFRASTRUCTURE ONLY: the CPU oracle for the GPU interior-point engine.
 *
 * A plain-C restatement of the reference's CPU algorithms on this path (file:line citations in
 * ipm_oracle.c). It is the checker for tests/, the smoke check and the CPU-baseline leg of
 * bench.py; the product library never links or calls it.
 *
 * Parity pin: tests/test_oracle.py checks every function here against the reference itself,
 * compiled unmodified into oracle/_ref/libsovref.so (oracle/Makefile), and against the golden
 * vectors under tests/golden/ that the reference produced (tests/golden/make_golden.py). */
#ifndef SOV_IPM_ORACLE_H
#define SOV_IPM_ORACLE_H

#include "sov_ipm.h"

#ifdef __cplusplus
extern "C" {
#endif

/* InteriorPointSolver::solve with the dense normal equations
 * (SOVEREIGN_IPM_NORMAL_EQUATIONS=dense). Returns 0. */
int oracle_lp_solve(const sov_model* model, const sov_options* opt, sov_result* result);

/* QpInteriorPointSolver's generic path: build_qp_form + solve_qp_ipm from the default start, then
 * from Mehrotra's start (qp_interior_point.cpp:3162-3179), dense KKT (SOVEREIGN_QP_KKT=dense). */
int oracle_qp_solve(const sov_model* model, const sov_options* opt, sov_result* result);

/* spmv_csc_cpu / spmv_csc_transpose_cpu (gpu_spmv.cpp:36-67). */
void oracle_spmv_csc(int32_t nrows, int32_t ncols, const int32_t* col_ptr, const int32_t* row_idx,
                     const double* values, const double* x, double* y, int32_t transpose);

/* build_normal_eq + DenseLU::factorize + DenseLU::solve (interior_point.cpp:74-101,
 * dense_lu.cpp:9-80) for nrhs column-major right-hand sides. Returns 0, or 1 when the LU pivot
 * floor (1e-14) rejects the matrix. */
int oracle_normal_factor_solve(int32_t m, int32_t n, const int32_t* col_ptr, const int32_t* row_idx,
                               const double* values, const double* d, double* rhs, int32_t nrhs);

/* The internal standard form (build_ipm_form, interior_point.cpp:224-409) as arrays, for tests of
 * the engine's host-side conversion. Sizes from sov_ipm_dims semantics; col_ptr has n_ipm + 1
 * entries, row_idx/values up to nnz_cap entries. Returns nnz or -1 when nnz_cap is too small. */
int oracle_ipm_form(const sov_model* model, int32_t enable_scaling, int32_t* col_ptr,
                    int32_t* row_idx, double* values, int32_t nnz_cap, double* b, double* c,
                    double* col_scale, double* row_scale, double* shift);

#ifdef __cplusplus
}
#endif

#endif
