/* ipm_oracle.c -- TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's interior-point
 * path, used as the checker of the GPU engine (never shipped, never called by the product).
 *
 * Restates, from the Abhishekmishra2808/sovereign sources:
 *   build_ipm_form          solver/lp/src/interior_point.cpp:224-409
 *   solve_ipm / publish     solver/lp/src/interior_point.cpp:454-740, 521-569
 *   solve_newton            solver/lp/src/interior_point.cpp:418-452
 *   build_normal_eq         solver/lp/src/interior_point.cpp:74-101
 *   DenseLU                 solver/numerical/src/dense_lu.cpp:9-80
 *   spmv_csc_cpu (+ A')     solver/gpu/src/gpu_spmv.cpp:36-67
 *   build_qp_form           solver/qp/src/qp_interior_point.cpp:119-250 (+ build_hessian :68-106)
 *   QpKkt dense path        solver/qp/src/qp_interior_point.cpp:449-479,583-603
 *   solve_qp_ipm            solver/qp/src/qp_interior_point.cpp:2827-3116
 *   QP dispatcher retry     solver/qp/src/qp_interior_point.cpp:3162-3179
 * The normal equations are always factored dense here (the reference's
 * SOVEREIGN_IPM_NORMAL_EQUATIONS=dense / SOVEREIGN_QP_KKT=dense paths); the reference's sparse
 * LDL^T path computes the same Newton directions up to rounding. */
#include "ipm_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ALLOC(T, n) ((T*)calloc((size_t)((n) > 0 ? (n) : 1), sizeof(T)))

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }
static double max_abs(const double* v, int n) {
  double m = 0.0;
  for (int i = 0; i < n; ++i) m = dmax(m, fabs(v[i]));
  return m;
}
static double dot(const double* a, const double* b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

/* ---------------------------------------------------------------------------------------- */
/* CSC container                                                                             */
/* ---------------------------------------------------------------------------------------- */
typedef struct {
  int m, n;
  int* col_ptr;
  int* row_idx;
  double* val;
} csc_t;

static void csc_free(csc_t* a) {
  free(a->col_ptr);
  free(a->row_idx);
  free(a->val);
}

/* gpu_spmv.cpp:36-51 (y = A x, column scatter) and :54-67 (y = A' x, column gather). */
static void csc_mul(const csc_t* A, const double* x, double* y) {
  for (int i = 0; i < A->m; ++i) y[i] = 0.0;
  for (int j = 0; j < A->n; ++j) {
    const double xj = x[j];
    if (xj == 0.0) continue;
    for (int p = A->col_ptr[j]; p < A->col_ptr[j + 1]; ++p) y[A->row_idx[p]] += A->val[p] * xj;
  }
}
static void csc_mul_t(const csc_t* A, const double* x, double* y) {
  for (int j = 0; j < A->n; ++j) {
    double s = 0.0;
    for (int p = A->col_ptr[j]; p < A->col_ptr[j + 1]; ++p) s += A->val[p] * x[A->row_idx[p]];
    y[j] = s;
  }
}

void oracle_spmv_csc(int32_t nrows, int32_t ncols, const int32_t* col_ptr, const int32_t* row_idx,
                     const double* values, const double* x, double* y, int32_t transpose) {
  csc_t A = {nrows, ncols, (int*)col_ptr, (int*)row_idx, (double*)values};
  if (transpose) csc_mul_t(&A, x, y);
  else csc_mul(&A, x, y);
}

/* ---------------------------------------------------------------------------------------- */
/* DenseLU (dense_lu.cpp:9-80): partial pivoting, column-major, pivot floor 1e-14             */
/* ---------------------------------------------------------------------------------------- */
typedef struct {
  int n;
  double* lu;
  int* piv;
} dense_lu_t;

static int lu_factorize(dense_lu_t* f) {
  const int n = f->n;
  double* a = f->lu;
  for (int i = 0; i < n; ++i) f->piv[i] = i;
  for (int k = 0; k < n; ++k) {
    int pr = k;
    double best = fabs(a[(size_t)k * n + k]);
    for (int i = k + 1; i < n; ++i) {
      const double v = fabs(a[(size_t)k * n + i]);
      if (v > best) {
        best = v;
        pr = i;
      }
    }
    if (best < 1e-14) return 0; /* dense_lu.cpp:32 */
    if (pr != k) {
      for (int j = 0; j < n; ++j) {
        double t = a[(size_t)j * n + k];
        a[(size_t)j * n + k] = a[(size_t)j * n + pr];
        a[(size_t)j * n + pr] = t;
      }
      int t = f->piv[k];
      f->piv[k] = f->piv[pr];
      f->piv[pr] = t;
    }
    const double akk = a[(size_t)k * n + k];
    for (int i = k + 1; i < n; ++i) {
      a[(size_t)k * n + i] /= akk;
      const double lik = a[(size_t)k * n + i];
      for (int j = k + 1; j < n; ++j) a[(size_t)j * n + i] -= lik * a[(size_t)j * n + k];
    }
  }
  return 1;
}

static void lu_solve(const dense_lu_t* f, double* x, double* work) {
  const int n = f->n;
  const double* a = f->lu;
  for (int i = 0; i < n; ++i) work[i] = x[f->piv[i]];
  for (int i = 0; i < n; ++i) {
    double s = work[i];
    for (int j = 0; j < i; ++j) s -= a[(size_t)j * n + i] * work[j];
    work[i] = s;
  }
  for (int ii = 0; ii < n; ++ii) {
    const int i = n - 1 - ii;
    double s = work[i];
    for (int j = i + 1; j < n; ++j) s -= a[(size_t)j * n + i] * work[j];
    work[i] = s / a[(size_t)i * n + i];
  }
  memcpy(x, work, sizeof(double) * (size_t)n);
}

/* build_normal_eq (interior_point.cpp:74-101): M = A diag(d) A', column-major, + 1e-12 diag. */
static void build_normal_eq(const csc_t* A, const double* d, double* M) {
  const int m = A->m;
  memset(M, 0, sizeof(double) * (size_t)m * (size_t)m);
  for (int j = 0; j < A->n; ++j) {
    const double dj = d[j];
    if (dj == 0.0) continue;
    for (int p = A->col_ptr[j]; p < A->col_ptr[j + 1]; ++p) {
      const int r = A->row_idx[p];
      const double ar = A->val[p] * dj;
      for (int q = A->col_ptr[j]; q < A->col_ptr[j + 1]; ++q) {
        M[(size_t)A->row_idx[q] * m + r] += ar * A->val[q];
      }
    }
  }
  for (int i = 0; i < m; ++i) M[(size_t)i * m + i] += 1e-12;
}

int oracle_normal_factor_solve(int32_t m, int32_t n, const int32_t* col_ptr, const int32_t* row_idx,
                               const double* values, const double* d, double* rhs, int32_t nrhs) {
  csc_t A = {m, n, (int*)col_ptr, (int*)row_idx, (double*)values};
  dense_lu_t f = {m, ALLOC(double, (size_t)m * m), ALLOC(int, m)};
  double* work = ALLOC(double, m);
  build_normal_eq(&A, d, f.lu);
  int ok = lu_factorize(&f);
  if (ok)
    for (int r = 0; r < nrhs; ++r) lu_solve(&f, rhs + (size_t)r * m, work);
  free(f.lu);
  free(f.piv);
  free(work);
  return ok ? 0 : 1;
}

/* ---------------------------------------------------------------------------------------- */
/* Column assembly shared by the LP and QP standard forms                                   */
/* ---------------------------------------------------------------------------------------- */
typedef struct {
  int row;
  double val;
} entry_t;

static int entry_cmp(const void* a, const void* b) {
  const entry_t* x = (const entry_t*)a;
  const entry_t* y = (const entry_t*)b;
  if (x->row != y->row) return x->row < y->row ? -1 : 1;
  return x->val < y->val ? -1 : (x->val > y->val ? 1 : 0);
}

/* Standard form of an index-form model: shift by lb, one Le row per finite upper bound, one
 * slack (+1, Le) or surplus (-1, Ge) column per inequality row, columns sorted by row with
 * duplicates merged and exact zeros dropped (interior_point.cpp:224-364 for the LP,
 * qp_interior_point.cpp:119-250 for the QP, which differs only in free columns). */
typedef struct {
  csc_t A;
  double* b;
  double* c;
  double* shift;     /* n_structural */
  double* col_scale; /* n */
  double* row_scale; /* m */
  char* free_col;    /* n (QP) */
  int n_struct, m0, m, n;
  double coef_min_before, coef_max_before, coef_min_after, coef_max_after;
  int scaling_applied;
} std_form_t;

static void std_form_free(std_form_t* f) {
  csc_free(&f->A);
  free(f->b);
  free(f->c);
  free(f->shift);
  free(f->col_scale);
  free(f->row_scale);
  free(f->free_col);
}

static void coefficient_range(const double* v, int nnz, double* mn, double* mx) {
  /* interior_point.cpp:46-56 */
  double lo = INFINITY, hi = 0.0;
  for (int p = 0; p < nnz; ++p) {
    const double a = fabs(v[p]);
    if (a == 0.0 || !isfinite(a)) continue;
    lo = dmin(lo, a);
    hi = dmax(hi, a);
  }
  if (!isfinite(lo)) lo = 0.0;
  *mn = lo;
  *mx = hi;
}

/* qp = 0: LP rules (every column shifted by lb). qp = 1: QP rules (lb <= -1e29 -> free column,
 * shift 0). Returns 0, or -1 with msg set for inconsistent bounds. */
static int build_std_form(const sov_model* p, int qp, int enable_scaling, std_form_t* f, char* msg,
                          size_t msglen) {
  memset(f, 0, sizeof(*f));
  const int ns = p->n, m0 = p->m;
  f->n_struct = ns;
  f->m0 = m0;
  f->shift = ALLOC(double, ns);
  char* free_s = ALLOC(char, ns);
  int* ub_var = ALLOC(int, ns);
  double* ub_val = ALLOC(double, ns);
  int n_ub = 0;
  for (int j = 0; j < ns; ++j) {
    const double lb = p->lb ? p->lb[j] : 0.0;
    const double ub = p->ub ? p->ub[j] : 1e30;
    const int no_lower = qp && !(lb > -1e29);
    free_s[j] = (char)no_lower;
    f->shift[j] = no_lower ? 0.0 : lb;
    if (isfinite(ub) && ub < 1e29) { /* interior_point.cpp:239 */
      const double u = ub - f->shift[j];
      if (!no_lower && u < -1e-12) {
        snprintf(msg, msglen, "Inconsistent bounds for variable x%d", j);
        free(free_s);
        free(ub_var);
        free(ub_val);
        return -1;
      }
      ub_var[n_ub] = j;
      ub_val[n_ub] = u;
      ++n_ub;
    }
  }
  const int m = m0 + n_ub;
  int n_slack = 0;
  for (int r = 0; r < m0; ++r)
    if (p->sense[r] != SOV_EQ) ++n_slack;
  n_slack += n_ub;
  const int n = ns + n_slack;
  f->m = m;
  f->n = n;
  f->b = ALLOC(double, m);
  f->c = ALLOC(double, n);
  f->col_scale = ALLOC(double, n);
  f->row_scale = ALLOC(double, m);
  f->free_col = ALLOC(char, n);
  for (int j = 0; j < ns; ++j) f->free_col[j] = free_s[j];
  for (int j = 0; j < n; ++j) f->col_scale[j] = 1.0;
  for (int i = 0; i < m; ++i) f->row_scale[i] = 1.0;

  /* rows: rhs minus a*shift (interior_point.cpp:276-293); merged per (row, column) first, like
   * the name-keyed map of a Constraint. */
  const int nnz_in = p->col_ptr[ns];
  int cap = nnz_in + n_ub + n_slack;
  entry_t* ent = ALLOC(entry_t, cap);
  int* cp = ALLOC(int, n + 1);
  int pos = 0;
  for (int i = 0; i < m0; ++i) f->b[i] = p->rhs[i];
  for (int j = 0; j < ns; ++j) {
    cp[j] = pos;
    const int start = pos;
    for (int k = p->col_ptr[j]; k < p->col_ptr[j + 1]; ++k) {
      ent[pos].row = p->row_idx[k];
      ent[pos].val = p->values[k];
      ++pos;
    }
    for (int k = 0; k < n_ub; ++k)
      if (ub_var[k] == j) {
        ent[pos].row = m0 + k;
        ent[pos].val = 1.0;
        ++pos;
      }
    /* sort by row and merge duplicates (interior_point.cpp:352-362) */
    qsort(ent + start, (size_t)(pos - start), sizeof(entry_t), entry_cmp);
    int w = start;
    for (int q = start; q < pos; ++q) {
      if (w > start && ent[w - 1].row == ent[q].row) ent[w - 1].val += ent[q].val;
      else ent[w++] = ent[q];
    }
    pos = w;
    for (int q = start; q < pos; ++q)
      if (ent[q].row < m0) f->b[ent[q].row] -= ent[q].val * f->shift[j];
  }
  for (int k = 0; k < n_ub; ++k) f->b[m0 + k] = ub_val[k];
  /* slack / surplus columns in row order (interior_point.cpp:339-350) */
  int sc = ns;
  for (int r = 0; r < m; ++r) {
    const int kind = r < m0 ? p->sense[r] : SOV_LE;
    if (kind == SOV_EQ) continue;
    cp[sc] = pos;
    ent[pos].row = r;
    ent[pos].val = kind == SOV_LE ? 1.0 : -1.0;
    ++pos;
    ++sc;
  }
  cp[n] = pos;
  /* drop exact zeros */
  f->A.m = m;
  f->A.n = n;
  f->A.col_ptr = ALLOC(int, n + 1);
  f->A.row_idx = ALLOC(int, pos);
  f->A.val = ALLOC(double, pos);
  int nnz = 0;
  for (int j = 0; j < n; ++j) {
    f->A.col_ptr[j] = nnz;
    for (int q = cp[j]; q < cp[j + 1]; ++q)
      if (fabs(ent[q].val) > 0.0) {
        f->A.row_idx[nnz] = ent[q].row;
        f->A.val[nnz] = ent[q].val;
        ++nnz;
      }
  }
  f->A.col_ptr[n] = nnz;
  free(ent);
  free(cp);
  free(free_s);
  free(ub_var);
  free(ub_val);

  /* objective, minimization sense (interior_point.cpp:321-329) */
  const double sign = p->maximize ? -1.0 : 1.0;
  for (int j = 0; j < ns; ++j) f->c[j] = sign * (p->obj ? p->obj[j] : 0.0);

  coefficient_range(f->A.val, nnz, &f->coef_min_before, &f->coef_max_before);
  f->scaling_applied = enable_scaling && m > 0 && n > 0;
  if (f->scaling_applied) { /* two passes of 1/sqrt(max|a|), rows then columns (:370-405) */
    double* row_max = ALLOC(double, m);
    for (int pass = 0; pass < 2; ++pass) {
      for (int i = 0; i < m; ++i) row_max[i] = 0.0;
      for (int q = 0; q < nnz; ++q) row_max[f->A.row_idx[q]] = dmax(row_max[f->A.row_idx[q]], fabs(f->A.val[q]));
      for (int i = 0; i < m; ++i) {
        const double rs = row_max[i] > 0.0 ? 1.0 / sqrt(row_max[i]) : 1.0;
        row_max[i] = rs;
        f->row_scale[i] *= rs;
        f->b[i] *= rs;
      }
      for (int q = 0; q < nnz; ++q) f->A.val[q] *= row_max[f->A.row_idx[q]];
      for (int j = 0; j < n; ++j) {
        double mx = 0.0;
        for (int q = f->A.col_ptr[j]; q < f->A.col_ptr[j + 1]; ++q) mx = dmax(mx, fabs(f->A.val[q]));
        const double s = mx > 0.0 ? 1.0 / sqrt(mx) : 1.0;
        for (int q = f->A.col_ptr[j]; q < f->A.col_ptr[j + 1]; ++q) f->A.val[q] *= s;
        f->c[j] *= s;
        f->col_scale[j] *= s;
      }
    }
    free(row_max);
  }
  coefficient_range(f->A.val, nnz, &f->coef_min_after, &f->coef_max_after);
  return 0;
}

int oracle_ipm_form(const sov_model* model, int32_t enable_scaling, int32_t* col_ptr,
                    int32_t* row_idx, double* values, int32_t nnz_cap, double* b, double* c,
                    double* col_scale, double* row_scale, double* shift) {
  std_form_t f;
  char msg[256];
  if (build_std_form(model, 0, enable_scaling, &f, msg, sizeof msg) != 0) return -1;
  const int nnz = f.A.col_ptr[f.n];
  if (nnz > nnz_cap) {
    std_form_free(&f);
    return -1;
  }
  memcpy(col_ptr, f.A.col_ptr, sizeof(int) * (size_t)(f.n + 1));
  memcpy(row_idx, f.A.row_idx, sizeof(int) * (size_t)nnz);
  memcpy(values, f.A.val, sizeof(double) * (size_t)nnz);
  memcpy(b, f.b, sizeof(double) * (size_t)f.m);
  memcpy(c, f.c, sizeof(double) * (size_t)f.n);
  memcpy(col_scale, f.col_scale, sizeof(double) * (size_t)f.n);
  memcpy(row_scale, f.row_scale, sizeof(double) * (size_t)f.m);
  memcpy(shift, f.shift, sizeof(double) * (size_t)f.n_struct);
  std_form_free(&f);
  return nnz;
}

/* ---------------------------------------------------------------------------------------- */
/* LP interior point (interior_point.cpp:411-740)                                             */
/* ---------------------------------------------------------------------------------------- */
static double step_to_bound(const double* x, const double* dx, const char* free_col, int n) {
  /* interior_point.cpp:214-222 (free_col NULL) / qp_interior_point.cpp:110-117 */
  double a = 1.0;
  for (int i = 0; i < n; ++i)
    if ((!free_col || !free_col[i]) && dx[i] < 0.0) a = dmin(a, -x[i] / dx[i]);
  return a;
}

typedef struct {
  const csc_t* A;
  dense_lu_t lu;
  double* work;
  int factorizations;
} normal_t;

static int normal_factor(normal_t* ne, const double* d) {
  build_normal_eq(ne->A, d, ne->lu.lu);
  ++ne->factorizations;
  return lu_factorize(&ne->lu);
}

/* solve_newton (interior_point.cpp:418-452) */
static void solve_newton(const csc_t* A, normal_t* ne, const double* d, const double* s,
                         const double* rp, const double* rd, const double* rxs, double* dx,
                         double* dy, double* ds, double* tmp_n, double* tmp_m) {
  const int n = A->n, m = A->m;
  for (int j = 0; j < n; ++j) tmp_n[j] = d[j] * rd[j] - rxs[j] / dmax(s[j], 1e-16);
  csc_mul(A, tmp_n, tmp_m);
  for (int i = 0; i < m; ++i) dy[i] = rp[i] + tmp_m[i];
  lu_solve(&ne->lu, dy, ne->work);
  csc_mul_t(A, dy, tmp_n);
  for (int j = 0; j < n; ++j) {
    dx[j] = d[j] * (tmp_n[j] - rd[j]) + rxs[j] / dmax(s[j], 1e-16);
    ds[j] = rd[j] - tmp_n[j];
  }
}

static void publish_lp(const sov_model* p, const std_form_t* f, const double* x, const double* y,
                       const double* s, int status, int iteration, double gap, double pres,
                       double dres, const char* message, sov_result* r) {
  /* publish_iterate (interior_point.cpp:521-569) */
  r->status = status;
  r->iterations = iteration;
  r->duality_gap = gap;
  r->primal_residual = pres;
  r->dual_residual = dres;
  r->has_objective_value = 1;
  double obj = p->obj_constant;
  for (int j = 0; j < f->n_struct; ++j) {
    const double v = f->shift[j] + f->col_scale[j] * x[j];
    if (r->primal) r->primal[j] = v;
    if (r->dual_col) r->dual_col[j] = s[j] / f->col_scale[j];
    obj += (p->obj ? p->obj[j] : 0.0) * v;
  }
  if (r->dual_row)
    for (int i = 0; i < f->m0; ++i) r->dual_row[i] = f->row_scale[i] * y[i];
  if (r->ipm_x) memcpy(r->ipm_x, x, sizeof(double) * (size_t)f->n);
  if (r->ipm_s) memcpy(r->ipm_s, s, sizeof(double) * (size_t)f->n);
  if (r->ipm_y) memcpy(r->ipm_y, y, sizeof(double) * (size_t)f->m);
  r->objective_value = obj;
  snprintf(r->message, sizeof(r->message), "%s", message);
}

int oracle_lp_solve(const sov_model* p, const sov_options* opt, sov_result* r) {
  r->status = SOV_ERROR;
  r->iterations = 0;
  r->has_objective_value = 0;
  std_form_t f;
  char msg[512];
  if (build_std_form(p, 0, opt->enable_scaling, &f, msg, sizeof msg) != 0) {
    snprintf(r->message, sizeof(r->message), "IPM error: %s", msg);
    return 0;
  }
  const int m = f.m, n = f.n;
  r->n_ipm = n;
  r->m_ipm = m;
  sov_diagnostics* dg = r->diagnostics;
  if (dg) {
    memset(dg, 0, sizeof(*dg));
    dg->scaling_applied = f.scaling_applied;
    dg->coefficient_min_abs_before = f.coef_min_before;
    dg->coefficient_max_abs_before = f.coef_max_before;
    dg->coefficient_min_abs_after = f.coef_min_after;
    dg->coefficient_max_abs_after = f.coef_max_after;
    dg->stall_iteration = -1;
  }
  if (n <= 0) {
    snprintf(r->message, sizeof(r->message), "IPM: empty model.");
    std_form_free(&f);
    return 0;
  }
  if (m <= 0) { /* interior_point.cpp:464-478 */
    r->status = SOV_OPTIMAL;
    r->has_objective_value = 1;
    double obj = p->obj_constant;
    for (int j = 0; j < f.n_struct; ++j) {
      if (r->primal) r->primal[j] = f.shift[j];
      obj += (p->obj ? p->obj[j] : 0.0) * f.shift[j];
    }
    r->objective_value = obj;
    snprintf(r->message, sizeof(r->message), "Optimal (no constraints) via IPM path.");
    std_form_free(&f);
    return 0;
  }
  const csc_t* A = &f.A;
  double *x = ALLOC(double, n), *s = ALLOC(double, n), *y = ALLOC(double, m);
  double *bx = ALLOC(double, n), *bs = ALLOC(double, n), *by = ALLOC(double, m);
  double *rp = ALLOC(double, m), *rd = ALLOC(double, n), *d = ALLOC(double, n);
  double *rxs = ALLOC(double, n), *tn = ALLOC(double, n), *tm = ALLOC(double, m);
  double *dxa = ALLOC(double, n), *dya = ALLOC(double, m), *dsa = ALLOC(double, n);
  double *dx = ALLOC(double, n), *dy = ALLOC(double, m), *ds = ALLOC(double, n);
  normal_t ne = {A, {m, ALLOC(double, (size_t)m * m), ALLOC(int, m)}, ALLOC(double, m), 0};
  for (int j = 0; j < n; ++j) x[j] = s[j] = 1.0;

  /* Mehrotra-like start (interior_point.cpp:488-506) */
  for (int j = 0; j < n; ++j) tn[j] = 1.0;
  if (normal_factor(&ne, tn)) {
    csc_mul(A, tn, tm);
    for (int i = 0; i < m; ++i) dy[i] = f.b[i] - tm[i];
    lu_solve(&ne.lu, dy, ne.work);
    csc_mul_t(A, dy, tn);
    for (int j = 0; j < n; ++j) {
      x[j] = dmax(1.0, fabs(tn[j]));
      s[j] = dmax(1.0, fabs(f.c[j] - tn[j]));
    }
    memcpy(y, dy, sizeof(double) * (size_t)m);
  }
  const double bnorm = dmax(1.0, max_abs(f.b, m));
  const double cnorm = dmax(1.0, max_abs(f.c, n));
  const double tau = opt->fraction_to_boundary;
  memcpy(bx, x, sizeof(double) * (size_t)n);
  memcpy(bs, s, sizeof(double) * (size_t)n);
  memcpy(by, y, sizeof(double) * (size_t)m);
  double best_metric = INFINITY, best_gap = INFINITY, best_p = INFINITY, best_d = INFINITY;
  int best_it = 0, stale = 0, done = 0, last_it = 0;
  const char* fail = NULL;

  for (int it = 0; it < opt->max_iterations && !done; ++it) {
    csc_mul(A, x, tm);
    for (int i = 0; i < m; ++i) rp[i] = f.b[i] - tm[i];
    csc_mul_t(A, y, tn);
    for (int j = 0; j < n; ++j) rd[j] = f.c[j] - (tn[j] + s[j]);
    const double xs = dot(x, s, n);
    const double mu = xs / (double)n;
    const double pres = max_abs(rp, m) / bnorm;
    const double dres = max_abs(rd, n) / cnorm;
    const double cx = dot(f.c, x, n);
    const double gap = fabs(xs) / (1.0 + fabs(cx)); /* interior_point.cpp:600-601 */
    const double metric = dmax(pres, dmax(dres, gap));
    if (metric < best_metric) {
      best_metric = metric;
      memcpy(bx, x, sizeof(double) * (size_t)n);
      memcpy(bs, s, sizeof(double) * (size_t)n);
      memcpy(by, y, sizeof(double) * (size_t)m);
      best_gap = gap;
      best_p = pres;
      best_d = dres;
      best_it = it + 1;
      stale = 0;
    } else {
      ++stale;
    }
    const int sample = it < 8 || it % 10 == 0 || it + 1 == opt->max_iterations;
    if (dg && sample && dg->history_len < SOV_HISTORY_MAX) {
      dg->history_iterations[dg->history_len] = it + 1;
      dg->objective_history[dg->history_len] = cx;
      dg->gap_history[dg->history_len] = gap;
      dg->mu_history[dg->history_len] = mu;
      dg->history_len++;
    }
    if (gap < best_gap) {
      best_gap = gap;
      stale = 0;
    } else if (stale >= 8 && dg && dg->stall_iteration < 0) {
      dg->stall_iteration = it + 1;
      dg->stall_gap = gap;
      dg->stall_mu = mu;
    }
    if (pres < opt->feasibility_tol && dres < opt->feasibility_tol && gap < opt->optimality_tol) {
      snprintf(msg, sizeof msg,
               "Optimal solution found by primal-dual interior-point (Mehrotra). Normal equations: "
               "dense LU (%d x %d).", m, m);
      publish_lp(p, &f, x, y, s, SOV_OPTIMAL, it + 1, gap, pres, dres, msg, r);
      done = 1;
      break;
    }
    for (int j = 0; j < n; ++j) {
      rxs[j] = -x[j] * s[j];
      d[j] = dmax(x[j], 1e-16) / dmax(s[j], 1e-16); /* scaling_diagonal :411-415 */
    }
    if (!normal_factor(&ne, d)) {
      fail = "IPM stopped because the affine predictor factorization failed; the best iterate is "
             "returned with optimality unproven.";
      break;
    }
    solve_newton(A, &ne, d, s, rp, rd, rxs, dxa, dya, dsa, tn, tm);
    const double ap_aff = step_to_bound(x, dxa, NULL, n);
    const double ad_aff = step_to_bound(s, dsa, NULL, n);
    double mu_aff = 0.0;
    for (int j = 0; j < n; ++j) mu_aff += (x[j] + ap_aff * dxa[j]) * (s[j] + ad_aff * dsa[j]);
    mu_aff /= (double)n;
    const double sigma = mu > 0.0 ? dmin(1.0, pow(mu_aff / mu, 3.0)) : 0.0;
    for (int j = 0; j < n; ++j) rxs[j] = -x[j] * s[j] - dxa[j] * dsa[j] + sigma * mu;
    solve_newton(A, &ne, d, s, rp, rd, rxs, dx, dy, ds, tn, tm);
    double ap = dmin(1.0, tau * step_to_bound(x, dx, NULL, n));
    double ad = dmin(1.0, tau * step_to_bound(s, ds, NULL, n));
    if (dg && sample && dg->step_history_len < SOV_HISTORY_MAX) {
      dg->primal_step_history[dg->step_history_len] = ap;
      dg->dual_step_history[dg->step_history_len] = ad;
      dg->step_history_len++;
    }
    if (dg && dg->stall_iteration == it + 1) {
      dg->stall_primal_step = ap;
      dg->stall_dual_step = ad;
    }
    for (int j = 0; j < n; ++j) {
      x[j] = dmax(x[j] + ap * dx[j], 1e-14);
      s[j] = dmax(s[j] + ad * ds[j], 1e-14);
    }
    for (int i = 0; i < m; ++i) y[i] += ad * dy[i];
    last_it = it + 1;
  }
  (void)last_it;
  if (!done) {
    const int st = best_p <= opt->feasibility_tol ? SOV_FEASIBLE : SOV_NUMERICAL_ERROR;
    if (fail) {
      publish_lp(p, &f, bx, by, bs, st, best_it, best_gap, best_p, best_d, fail, r);
    } else {
      snprintf(msg, sizeof msg,
               "IPM stopped after %d iterations without meeting tolerance; returning best iterate "
               "from %d as a lower-accuracy candidate. Relative duality gap = %g (tolerance %g), "
               "primal residual = %g, dual residual = %g. Optimality is not proven.",
               opt->max_iterations, best_it, best_gap, opt->optimality_tol, best_p, best_d);
      publish_lp(p, &f, bx, by, bs, st, best_it, best_gap, best_p, best_d, msg, r);
    }
  }
  if (dg) dg->refactorizations = ne.factorizations;
  free(x); free(s); free(y); free(bx); free(bs); free(by); free(rp); free(rd); free(d);
  free(rxs); free(tn); free(tm); free(dxa); free(dya); free(dsa); free(dx); free(dy); free(ds);
  free(ne.lu.lu); free(ne.lu.piv); free(ne.work);
  std_form_free(&f);
  return 0;
}

/* ---------------------------------------------------------------------------------------- */
/* QP interior point, generic path (qp_interior_point.cpp:68-250, 449-479, 583-603,           */
/* 2827-3116, 3162-3179)                                                                      */
/* ---------------------------------------------------------------------------------------- */
typedef struct {
  std_form_t f;
  csc_t Q; /* both triangles, + 1e-14 on structural diagonal */
} qp_form_t;

static void qp_form_free(qp_form_t* q) {
  std_form_free(&q->f);
  csc_free(&q->Q);
}

/* build_hessian (qp_interior_point.cpp:68-106) */
static void build_hessian(const sov_model* p, int n_total, double sign, csc_t* Q) {
  const int ns = p->n;
  int cap = 2 * (p->q_col_ptr ? p->q_col_ptr[ns] : 0) + ns;
  int* cnt = ALLOC(int, n_total + 1);
  entry_t* e = ALLOC(entry_t, cap);
  int* col = ALLOC(int, cap);
  int k = 0;
  if (p->q_col_ptr) {
    for (int j = 0; j < ns; ++j)
      for (int q = p->q_col_ptr[j]; q < p->q_col_ptr[j + 1]; ++q) {
        const int i = p->q_row_idx[q];
        const double v = sign * p->q_values[q];
        if (i == j) {
          col[k] = i; e[k].row = i; e[k].val = v; ++k;
        } else {
          col[k] = j; e[k].row = i; e[k].val = 0.5 * v; ++k;
          col[k] = i; e[k].row = j; e[k].val = 0.5 * v; ++k;
        }
      }
  }
  for (int i = 0; i < ns; ++i) {
    col[k] = i; e[k].row = i; e[k].val = 1e-14; ++k;
  }
  /* bucket by column, then sort rows and merge */
  for (int q = 0; q < k; ++q) cnt[col[q] + 1]++;
  for (int j = 0; j < n_total; ++j) cnt[j + 1] += cnt[j];
  entry_t* b = ALLOC(entry_t, k);
  int* fill = ALLOC(int, n_total);
  for (int q = 0; q < k; ++q) b[cnt[col[q]] + fill[col[q]]++] = e[q];
  Q->m = Q->n = n_total;
  Q->col_ptr = ALLOC(int, n_total + 1);
  Q->row_idx = ALLOC(int, k);
  Q->val = ALLOC(double, k);
  int nnz = 0;
  for (int j = 0; j < n_total; ++j) {
    Q->col_ptr[j] = nnz;
    qsort(b + cnt[j], (size_t)(cnt[j + 1] - cnt[j]), sizeof(entry_t), entry_cmp);
    for (int q = cnt[j]; q < cnt[j + 1];) {
      const int r = b[q].row;
      double v = 0.0;
      for (; q < cnt[j + 1] && b[q].row == r; ++q) v += b[q].val;
      if (v != 0.0) {
        Q->row_idx[nnz] = r;
        Q->val[nnz] = v;
        ++nnz;
      }
    }
  }
  Q->col_ptr[n_total] = nnz;
  free(cnt); free(e); free(col); free(b); free(fill);
}

static void sym_mul(const csc_t* Q, const double* x, double* y) { csc_mul(Q, x, y); }

typedef struct {
  const qp_form_t* qp;
  int n, m, N;
  double* h;
  dense_lu_t lu;
  double* z;
  double* work;
  int with_hessian;
} qp_kkt_t;

/* factor_dense (qp_interior_point.cpp:583-603) after the h of factor (:449-456) */
static int kkt_factor(qp_kkt_t* k, const double* x, const double* s, int with_hessian) {
  const int n = k->n, m = k->m, N = k->N;
  const qp_form_t* qp = k->qp;
  k->with_hessian = with_hessian;
  for (int j = 0; j < n; ++j)
    k->h[j] = with_hessian ? (qp->f.free_col[j] ? 0.0 : dmax(s[j], 1e-16) / dmax(x[j], 1e-16)) : 1.0;
  double* K = k->lu.lu;
  memset(K, 0, sizeof(double) * (size_t)N * (size_t)N);
  for (int j = 0; j < n; ++j) {
    if (with_hessian)
      for (int q = qp->Q.col_ptr[j]; q < qp->Q.col_ptr[j + 1]; ++q)
        K[(size_t)j * N + qp->Q.row_idx[q]] += qp->Q.val[q];
    K[(size_t)j * N + j] += k->h[j];
    for (int q = qp->f.A.col_ptr[j]; q < qp->f.A.col_ptr[j + 1]; ++q) {
      const int r = qp->f.A.row_idx[q];
      const double a = qp->f.A.val[q];
      K[(size_t)j * N + n + r] += a;
      K[(size_t)(n + r) * N + j] -= a;
    }
  }
  for (int i = n; i < N; ++i) K[(size_t)i * N + i] -= 1e-12;
  return lu_factorize(&k->lu);
}

static void kkt_solve(qp_kkt_t* k, const double* r1, const double* r2, double* dx, double* dy) {
  memcpy(k->z, r1, sizeof(double) * (size_t)k->n);
  memcpy(k->z + k->n, r2, sizeof(double) * (size_t)k->m);
  lu_solve(&k->lu, k->z, k->work);
  memcpy(dx, k->z, sizeof(double) * (size_t)k->n);
  memcpy(dy, k->z + k->n, sizeof(double) * (size_t)k->m);
}

static void publish_qp(const sov_model* p, const qp_form_t* qp, const double* x, const double* y,
                       const double* s, sov_result* r) {
  /* optimal branch (qp_interior_point.cpp:3018-3037) + capture_diagnostics (:2862-2877) */
  const std_form_t* f = &qp->f;
  double obj = p->obj_constant;
  double* prim = ALLOC(double, f->n_struct);
  for (int j = 0; j < f->n_struct; ++j) prim[j] = f->shift[j] + x[j];
  for (int j = 0; j < f->n_struct; ++j) obj += (p->obj ? p->obj[j] : 0.0) * prim[j];
  if (p->q_col_ptr)
    for (int j = 0; j < f->n_struct; ++j)
      for (int q = p->q_col_ptr[j]; q < p->q_col_ptr[j + 1]; ++q)
        obj += 0.5 * p->q_values[q] * prim[p->q_row_idx[q]] * prim[j];
  r->objective_value = obj;
  if (r->primal) memcpy(r->primal, prim, sizeof(double) * (size_t)f->n_struct);
  if (r->dual_col) memcpy(r->dual_col, s, sizeof(double) * (size_t)f->n_struct);
  if (r->dual_row) memcpy(r->dual_row, y, sizeof(double) * (size_t)f->m0);
  if (r->ipm_x) memcpy(r->ipm_x, x, sizeof(double) * (size_t)f->n);
  if (r->ipm_s) memcpy(r->ipm_s, s, sizeof(double) * (size_t)f->n);
  if (r->ipm_y) memcpy(r->ipm_y, y, sizeof(double) * (size_t)f->m);
  free(prim);
}

/* solve_qp_ipm (qp_interior_point.cpp:2848-3116) */
static void solve_qp_ipm(const sov_model* p, const qp_form_t* qp, const sov_options* opt,
                         int mehrotra_start, sov_result* r) {
  const std_form_t* f = &qp->f;
  const int n = f->n, m = f->m;
  const char* fr = f->free_col;
  r->has_objective_value = 0;
  if (n <= 0) {
    r->status = SOV_ERROR;
    snprintf(r->message, sizeof(r->message), "QP-IPM: empty model.");
    return;
  }
  double *x = ALLOC(double, n), *s = ALLOC(double, n), *y = ALLOC(double, m);
  double *rp = ALLOC(double, m), *rd = ALLOC(double, n), *Qx = ALLOC(double, n);
  double *tn = ALLOC(double, n), *tn2 = ALLOC(double, n), *tm = ALLOC(double, m);
  double *rxs = ALLOC(double, n), *r1 = ALLOC(double, n);
  double *dxa = ALLOC(double, n), *dya = ALLOC(double, m), *dsa = ALLOC(double, n);
  double *dx = ALLOC(double, n), *dy = ALLOC(double, m), *ds = ALLOC(double, n);
  qp_kkt_t k = {qp, n, m, n + m, ALLOC(double, n), {n + m, ALLOC(double, (size_t)(n + m) * (n + m)), ALLOC(int, n + m)},
                ALLOC(double, n + m), ALLOC(double, n + m), 1};
  for (int j = 0; j < n; ++j) x[j] = s[j] = 1.0;
  if (m > 0) {
    for (int j = 0; j < n; ++j) tn[j] = 1.0;
    if (kkt_factor(&k, tn, tn, 0)) {
      csc_mul(&f->A, tn, tm);
      double* r2 = ALLOC(double, m);
      double* zero = ALLOC(double, n);
      for (int i = 0; i < m; ++i) r2[i] = f->b[i] - tm[i];
      kkt_solve(&k, zero, r2, tn2, dy);
      csc_mul_t(&f->A, dy, tn); /* Atdy */
      if (mehrotra_start) {
        double* xt = ALLOC(double, n);
        double* zm = ALLOC(double, m);
        double* u = ALLOC(double, n);
        double* yls = ALLOC(double, m);
        for (int j = 0; j < n; ++j) xt[j] = 1.0 + tn[j];
        sym_mul(&qp->Q, xt, Qx);
        for (int j = 0; j < n; ++j) r1[j] = -(f->c[j] + Qx[j]);
        kkt_solve(&k, r1, zm, u, yls);
        double min_x = INFINITY, min_s = INFINITY;
        for (int j = 0; j < n; ++j) {
          if (fr[j]) continue;
          min_x = dmin(min_x, xt[j]);
          min_s = dmin(min_s, -u[j]);
        }
        const double sx = dmax(-1.5 * min_x, 0.0), ss = dmax(-1.5 * min_s, 0.0);
        double xs = 0.0, sum_x = 0.0, sum_s = 0.0;
        for (int j = 0; j < n; ++j) {
          if (fr[j]) continue;
          const double xh = xt[j] + sx, sh = -u[j] + ss;
          xs += xh * sh;
          sum_x += xh;
          sum_s += sh;
        }
        const double bx = sum_s > 0.0 ? 0.5 * xs / sum_s : 1.0;
        const double bs = sum_x > 0.0 ? 0.5 * xs / sum_x : 1.0;
        for (int j = 0; j < n; ++j) {
          if (fr[j]) {
            x[j] = xt[j];
            continue;
          }
          x[j] = dmax(1e-8, xt[j] + sx + bx);
          s[j] = dmax(1e-8, -u[j] + ss + bs);
        }
        memcpy(y, yls, sizeof(double) * (size_t)m);
        free(xt); free(zm); free(u); free(yls);
      } else {
        double* ones = ALLOC(double, n);
        for (int j = 0; j < n; ++j) ones[j] = 1.0;
        sym_mul(&qp->Q, ones, Qx);
        for (int j = 0; j < n; ++j) {
          if (fr[j]) {
            x[j] = 1.0 + tn[j];
            continue;
          }
          x[j] = dmax(1.0, fabs(tn[j]));
          s[j] = dmax(1.0, fabs(Qx[j] + f->c[j] - tn[j]));
        }
        memcpy(y, dy, sizeof(double) * (size_t)m);
        free(ones);
      }
      free(r2);
      free(zero);
    }
  }
  int nb = 0;
  for (int j = 0; j < n; ++j) {
    if (fr[j]) s[j] = 0.0;
    else ++nb;
  }
  const double cc = nb > 1 ? (double)nb : 1.0;
  int has_q = 0;
  for (int q = 0; q < qp->Q.col_ptr[n]; ++q) has_q |= fabs(qp->Q.val[q]) > 1e-12;
  const double bnorm = dmax(1.0, max_abs(f->b, m)), cnorm = dmax(1.0, max_abs(f->c, n));
  const double tau = opt->fraction_to_boundary;
  double offset;
  {
    double* sh = ALLOC(double, n);
    for (int j = 0; j < f->n_struct; ++j) sh[j] = f->shift[j];
    sym_mul(&qp->Q, sh, tn);
    offset = dot(f->c, sh, n) - 0.5 * dot(sh, tn, n) + (p->maximize ? -1.0 : 1.0) * p->obj_constant;
    free(sh);
  }
  int done = 0;
  r->iterations = 0;
  for (int it = 0; it < opt->max_iterations && !done; ++it) {
    csc_mul(&f->A, x, tm);
    for (int i = 0; i < m; ++i) rp[i] = f->b[i] - tm[i];
    sym_mul(&qp->Q, x, Qx);
    csc_mul_t(&f->A, y, tn);
    for (int j = 0; j < n; ++j) rd[j] = Qx[j] + f->c[j] - tn[j] - s[j];
    const double mu = dot(x, s, n) / cc;
    const double pres = max_abs(rp, m) / bnorm;
    const double dres = max_abs(rd, n) / dmax(1.0, cnorm + max_abs(Qx, n));
    const double gap = mu * cc / (1.0 + fabs(dot(f->c, x, n) + 0.5 * dot(x, Qx, n) + offset));
    r->duality_gap = gap;
    r->primal_residual = pres;
    r->dual_residual = dres;
    if (pres < opt->feasibility_tol && dres < opt->feasibility_tol && gap < opt->optimality_tol) {
      r->status = SOV_OPTIMAL;
      r->iterations = it + 1;
      r->has_objective_value = 1;
      snprintf(r->message, sizeof(r->message),
               "Optimal convex QP found by Mehrotra predictor-corrector IPM. KKT system: dense LU "
               "(%d x %d).", n + m, n + m);
      publish_qp(p, qp, x, y, s, r);
      done = 1;
      break;
    }
    if (!kkt_factor(&k, x, s, 1)) {
      r->status = SOV_ERROR;
      r->iterations = it;
      publish_qp(p, qp, x, y, s, r);
      r->has_objective_value = 0;
      snprintf(r->message, sizeof(r->message), "QP-IPM Newton factorization failed.");
      done = 1;
      break;
    }
    for (int j = 0; j < n; ++j) rxs[j] = -x[j] * s[j];
    for (int pass = 0; pass < 2; ++pass) {
      double* ddx = pass ? dx : dxa;
      double* ddy = pass ? dy : dya;
      double* dds = pass ? ds : dsa;
      /* solve_newton_qp (qp_interior_point.cpp:2827-2846) */
      for (int j = 0; j < n; ++j) r1[j] = fr[j] ? -rd[j] : -rd[j] + rxs[j] / dmax(x[j], 1e-16);
      kkt_solve(&k, r1, rp, ddx, ddy);
      for (int j = 0; j < n; ++j) dds[j] = fr[j] ? 0.0 : (rxs[j] - s[j] * ddx[j]) / dmax(x[j], 1e-16);
      if (pass == 0) {
        const double apa = step_to_bound(x, dxa, fr, n), ada = step_to_bound(s, dsa, fr, n);
        double mua = 0.0;
        for (int j = 0; j < n; ++j)
          if (!fr[j]) mua += (x[j] + apa * dxa[j]) * (s[j] + ada * dsa[j]);
        mua /= cc;
        const double sigma = mu > 0.0 ? dmin(1.0, pow(mua / mu, 3.0)) : 0.0;
        for (int j = 0; j < n; ++j) rxs[j] = fr[j] ? 0.0 : -x[j] * s[j] - dxa[j] * dsa[j] + sigma * mu;
      }
    }
    double ap = dmin(1.0, tau * step_to_bound(x, dx, fr, n));
    double ad = dmin(1.0, tau * step_to_bound(s, ds, fr, n));
    if (has_q) ap = ad = dmin(ap, ad); /* common step (:3095) */
    for (int j = 0; j < n; ++j) {
      if (fr[j]) {
        x[j] += ap * dx[j];
        continue;
      }
      x[j] = dmax(1e-14, x[j] + ap * dx[j]);
      s[j] = dmax(1e-14, s[j] + ad * ds[j]);
    }
    for (int i = 0; i < m; ++i) y[i] += ad * dy[i];
    r->iterations = it + 1;
  }
  if (!done) {
    r->status = SOV_ERROR;
    publish_qp(p, qp, x, y, s, r);
    r->has_objective_value = 0;
    snprintf(r->message, sizeof(r->message), "QP-IPM iteration limit reached without convergence.");
  }
  free(x); free(s); free(y); free(rp); free(rd); free(Qx); free(tn); free(tn2); free(tm);
  free(rxs); free(r1); free(dxa); free(dya); free(dsa); free(dx); free(dy); free(ds);
  free(k.h); free(k.lu.lu); free(k.lu.piv); free(k.z); free(k.work);
}

int oracle_qp_solve(const sov_model* p, const sov_options* opt, sov_result* r) {
  qp_form_t qp;
  char msg[256];
  memset(&qp, 0, sizeof qp);
  r->status = SOV_ERROR;
  if (build_std_form(p, 1, 0, &qp.f, msg, sizeof msg) != 0) {
    snprintf(r->message, sizeof(r->message), "QP-IPM error: %s", msg);
    return 0;
  }
  /* Q carries the minimization sign; c_eff = sense*c + Q*shift (qp_interior_point.cpp:204-216) */
  build_hessian(p, qp.f.n, p->maximize ? -1.0 : 1.0, &qp.Q);
  {
    double* sh = ALLOC(double, qp.f.n);
    double* qs = ALLOC(double, qp.f.n);
    for (int j = 0; j < qp.f.n_struct; ++j) sh[j] = qp.f.shift[j];
    csc_mul(&qp.Q, sh, qs);
    for (int j = 0; j < qp.f.n_struct; ++j) qp.f.c[j] += qs[j];
    free(sh);
    free(qs);
  }
  r->n_ipm = qp.f.n;
  r->m_ipm = qp.f.m;
  solve_qp_ipm(p, &qp, opt, 0, r);
  if (r->status != SOV_OPTIMAL) {
    const int first_it = r->iterations;
    char first_msg[512];
    snprintf(first_msg, sizeof first_msg, "%s", r->message);
    sov_result second = *r;
    solve_qp_ipm(p, &qp, opt, 1, &second);
    if (second.status == SOV_OPTIMAL) {
      *r = second;
      r->iterations += first_it;
    } else {
      /* first result stays, with the second message appended (:3178) -- the buffers already
       * hold the second attempt's point, which the reference would not publish; rerun first. */
      solve_qp_ipm(p, &qp, opt, 0, r);
      char joined[512];
      snprintf(joined, sizeof joined, "%s | Mehrotra starting point: %s", first_msg, second.message);
      snprintf(r->message, sizeof(r->message), "%s", joined);
    }
  }
  qp_form_free(&qp);
  return 0;
}
