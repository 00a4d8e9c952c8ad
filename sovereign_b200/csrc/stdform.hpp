// stdform.hpp -- host-side standard form of an LP / convex QP for the interior-point engine.
//
// Same semantics as the reference's conversions, written for index-form input:
//   LP  build_ipm_form  (solver/lp/src/interior_point.cpp:224-409): shift by lb, one Le row per
//       finite upper bound, slack (+1) / surplus (-1) columns, max -> min, columns sorted with
//       duplicates merged and zeros dropped, two passes of 1/sqrt(max|a|) row/column scaling.
//   QP  build_qp_form   (solver/qp/src/qp_interior_point.cpp:119-250) + build_hessian (:68-106):
//       columns without a lower bound are free (no barrier, shift 0), Q with both triangles
//       (off-diagonal stored terms halved into each triangle), +1e-14 on structural diagonals,
//       c_eff = sense * c + Q * shift, no scaling.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "sov_ipm.h"

namespace sov {

struct StdForm {
  bool qp = false;
  int n_struct = 0, m0 = 0, m = 0, n = 0;
  // A (scaled), CSC and CSR
  std::vector<int> col_ptr, row_idx;
  std::vector<double> val;
  std::vector<int> row_ptr, col_idx;
  std::vector<double> rval;
  std::vector<double> b, c, col_scale, row_scale, shift;
  std::vector<uint8_t> free_col;
  // QP Hessian over the IPM columns: both triangles, CSC; qdiag = its diagonal.
  std::vector<int> q_ptr, q_idx;
  std::vector<double> q_val, qdiag;
  bool q_diagonal = true;  // no off-diagonal entries
  bool has_quadratic = false;
  double objective_offset = 0.0;  // QP gap offset (qp_interior_point.cpp:2966-2975)
  // diagnostics (LpDiagnostics, types.hpp:64-69)
  bool scaling_applied = false;
  double coef_min_before = 0, coef_max_before = 0, coef_min_after = 0, coef_max_after = 0;

  int nnz() const { return static_cast<int>(val.size()); }
};

// Throws std::runtime_error with the reference's message for inconsistent bounds.
StdForm build_std_form(const sov_model& model, bool qp, bool enable_scaling);

// LP standard form written straight into caller-provided arrays, for LPs whose structural columns
// are "plain" (rows strictly increasing, no zero or NaN values: nothing to sort, merge or drop).
// The arrays receive bit for bit what build_std_form(model, false, scaling) would hold.
struct LpShape {
  int n_struct, m0, m, n, nnz, n_ub;
};
// false when some column is not plain (the caller then uses build_std_form)
bool plain_lp_shape(const sov_model& model, LpShape* shape);
struct LpFormOut {
  int* col_ptr;       // n + 1
  int* row_idx;       // nnz
  double* val;        // nnz
  int* row_ptr;       // m + 1
  int* col_idx;       // nnz
  double* rval;       // nnz
  double* b;          // m
  double* c;          // n
  double* shift;      // n_struct
  double* col_scale;  // n
  double* row_scale;  // m
};
struct LpFormInfo {
  bool scaling_applied;
  double coef_min_before, coef_max_before, coef_min_after, coef_max_after;
};
// with_rows false: the row-wise copy is left to the caller except its row starts (out.row_ptr),
// which are always written (the batched path fills col_idx / rval on the GPU)
void build_plain_lp_into(const sov_model& model, const LpShape& shape, bool enable_scaling, const LpFormOut& out,
                         LpFormInfo* info, bool with_rows = true);

// Lower-triangle pattern of M = A diag(d) A' as a gather map: target entry t (position in the
// caller's matrix layout, from `index(row, col)`) receives sum over its contributions
// w * d[col_of_w]. Built once per solve; each IPM iteration is then one pass over this map
// (interior_point.cpp:74-101 / sparse_symmetric.cpp:103-169 arithmetic, w = a_ik * a_jk).
struct AssemblyMap {
  std::vector<int64_t> target;  // ntargets, sorted
  std::vector<int> ptr;         // ntargets + 1
  std::vector<int> col;         // contributions: IPM column k
  std::vector<double> w;        // contributions: a_ik * a_jk
  std::vector<int> diag_target; // m: index into `target` of each diagonal entry
};

// Dense column-major (ld) or band (kd) layouts.
AssemblyMap build_assembly_dense(const StdForm& f, int ld);          // column-major: c * ld + r, r >= c
AssemblyMap build_assembly_rowmajor(const StdForm& f, int ld);       // row-major lower: r * ld + c, r >= c
AssemblyMap build_assembly_band(const StdForm& f, int kd);  // band storage: (kd+1) x m, row-major by diagonal offset

// Half-bandwidth of A D A' in the natural row order.
int normal_bandwidth(const StdForm& f);

// x-space form of a QP whose every row carries a slack column and whose structural columns all
// have Q_jj > 0: K = diag(Q_jj + h_j) + A_x' Theta A_x over the structural columns, Theta_r the
// barrier weight s/x of row r's slack column.
struct XSpace {
  bool eligible = false;
  std::vector<int> slack_of_row;  // m: IPM column of row r's slack
  std::vector<double> sigma;      // m: that slack's coefficient (+1 slack, -1 surplus)
  int kd = 0;                     // half-bandwidth of K in the natural column order
};
XSpace analyze_xspace(const StdForm& f);
// Gather map of A_x' Theta A_x (contribution weight column = the row's slack column).
AssemblyMap build_assembly_xspace(const StdForm& f, const XSpace& xs, int ld);   // dense, ld >= n_struct
AssemblyMap build_assembly_xspace_band(const StdForm& f, const XSpace& xs);     // band, (kd+1) x n_struct

}  // namespace sov
