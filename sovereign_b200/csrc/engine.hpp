// engine.hpp -- single-problem GPU interior-point engine (LP and diagonal-Hessian QP).
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "sov_ipm.h"
#include "stdform.hpp"

namespace sov {

struct EngineStats {
  int launches = 0;
  int factorizations = 0;
  int solves = 0;
  double kernel_ms = 0.0;      // device time of the iteration loop (CUDA events)
  double factor_flops = 0.0;   // algorithmic flops of all factorizations
  double bytes = 0.0;          // algorithmic HBM bytes of the vector passes
};

// Solves one standard-form problem on the current device. `model` is the original model (for
// publishing objective and name-indexed outputs). Never throws; errors land in `result`.
int solve_single(const sov_model& model, const StdForm& f, const sov_options& opt, sov_result* result,
                 cudaStream_t stream, EngineStats* stats);

}  // namespace sov
