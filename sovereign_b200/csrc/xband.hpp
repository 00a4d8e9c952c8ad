// xband.hpp -- x-space banded interior-point solver in double-double for separable convex QPs
// whose constraint rows are narrow bands (the convex-sequence / LISWET shape).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "engine.hpp"
#include "sov_ipm.h"

namespace sov {

constexpr int kXBandMaxKd = 4;  // widest row span (last column - first column) the path takes

// The model in the form the solver works on: min 1/2 x'Qx + c'x, Q = diag(q) > 0, x free, every
// row an inequality written as a_r x >= b_r (<= rows negated), A held both by rows and by columns.
struct XBandModel {
  int n = 0, m = 0, kd = 0;
  std::vector<int32_t> row_ptr, col_idx, col_ptr, row_idx;
  std::vector<double> row_val, col_val, q, c, b;
  std::vector<int8_t> row_sign;  // +1 for >= rows, -1 for <= rows (multipliers published with it)
  double obj_constant = 0.0;
};

// True when `model` is a minimisation QP with a positive diagonal Hessian, every variable free
// (no finite bound), every row an inequality and every row's columns within kXBandMaxKd of each
// other; fills `out`. SOVEREIGN_QP_DISABLE=xband turns the path off.
bool xband_prepare(const sov_model& model, XBandModel* out);

// Solves it on the current device, one persistent launch; fills `result` like the general engine
// (primal, row duals, objective, residuals, gap, iterations, message, diagnostics).
int solve_xband(const sov_model& model, const XBandModel& xb, const sov_options& opt, sov_result* result,
                cudaStream_t stream, EngineStats* stats);

}  // namespace sov
