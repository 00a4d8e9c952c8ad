// capi.cu -- the extern "C" boundary (include/sov_ipm.h).
//
// Errors never cross the boundary as exceptions: the reference converts every exception of a
// solve into SolverStatus::Error with "IPM error: ..." (interior_point.cpp:748-756,
// qp_interior_point.cpp:3180-3184); the entry points do the same and additionally return a
// negative code when the failure was the device's (no sm_100 GPU, a CUDA error).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch.hpp"
#include "common.cuh"
#include "dense.cuh"
#include "engine.hpp"
#include "family.cuh"
#include "ipm_kernels.cuh"
#include "sov_ipm.h"
#include "stdform.hpp"

namespace {

thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int check_device() {
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0)
    return set_error(SOV_E_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  int dev = 0, major = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
  if (major != 10) return set_error(SOV_E_NO_DEVICE, "the kernels are built for sm_100a (B200); device is sm_" +
                                                         std::to_string(major) + "x");
  return SOV_OK;
}

}  // namespace

namespace sov {
// The same error record and device check for entry points defined in other files.
int record_error(int code, const std::string& msg) { return set_error(code, msg); }
int require_device() { return check_device(); }
}  // namespace sov

namespace {

int validate(const sov_model* p) {
  if (!p) return set_error(SOV_E_ARGUMENT, "null model");
  if (p->n < 0 || p->m < 0) return set_error(SOV_E_ARGUMENT, "negative dimensions");
  if (p->n > 0 && (!p->col_ptr || (p->col_ptr[p->n] > 0 && (!p->row_idx || !p->values))))
    return set_error(SOV_E_ARGUMENT, "missing constraint matrix arrays");
  if (p->m > 0 && (!p->sense || !p->rhs)) return set_error(SOV_E_ARGUMENT, "missing row senses or right-hand sides");
  if (p->n > 0 && p->col_ptr[0] != 0) return set_error(SOV_E_ARGUMENT, "col_ptr[0] must be 0");
  for (int j = 0; j < p->n; ++j)
    if (p->col_ptr[j + 1] < p->col_ptr[j]) return set_error(SOV_E_ARGUMENT, "col_ptr is not monotone");
  const int nnz = p->n > 0 ? p->col_ptr[p->n] : 0;
  for (int k = 0; k < nnz; ++k)
    if (p->row_idx[k] < 0 || p->row_idx[k] >= p->m) return set_error(SOV_E_ARGUMENT, "row index out of range");
  for (int i = 0; i < p->m; ++i)
    if (p->sense[i] < SOV_LE || p->sense[i] > SOV_EQ) return set_error(SOV_E_ARGUMENT, "invalid row sense");
  if (p->q_col_ptr) {
    for (int j = 0; j < p->n; ++j)
      if (p->q_col_ptr[j + 1] < p->q_col_ptr[j]) return set_error(SOV_E_ARGUMENT, "q_col_ptr is not monotone");
    for (int k = 0; k < p->q_col_ptr[p->n]; ++k)
      if (p->q_row_idx[k] < 0 || p->q_row_idx[k] >= p->n) return set_error(SOV_E_ARGUMENT, "Q row index out of range");
  }
  return SOV_OK;
}

void reset_result(sov_result* r) {
  r->status = SOV_ERROR;
  r->iterations = 0;
  r->has_objective_value = 0;
  r->objective_value = r->duality_gap = r->primal_residual = r->dual_residual = 0.0;
  r->solve_seconds = 0.0;
  r->message[0] = '\0';
}

struct StreamGuard {
  cudaStream_t s = nullptr;
  StreamGuard() { SOV_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~StreamGuard() {
    if (s) cudaStreamDestroy(s);
  }
};

int solve_one(const sov_model* model, const sov_options* opt_in, sov_result* result, bool qp) {
  if (!result) return set_error(SOV_E_ARGUMENT, "null result");
  reset_result(result);
  int rc = validate(model);
  if (rc) {
    std::snprintf(result->message, sizeof(result->message), "%s error: %s", qp ? "QP-IPM" : "IPM",
                  g_last_error.c_str());
    return rc;
  }
  sov_options opt;
  if (opt_in) opt = *opt_in;
  else if (qp) sov_default_qp_options(&opt);
  else sov_default_lp_options(&opt);
  if (qp) opt.enable_scaling = 0;  // the QP path never scales (qp_interior_point.hpp:11)
  try {
    rc = check_device();
    if (rc) throw std::runtime_error(g_last_error);
    sov::StdForm f = sov::build_std_form(*model, qp, opt.enable_scaling != 0);
    result->n_ipm = f.n;
    result->m_ipm = f.m;
    if (f.n <= 0) {
      std::snprintf(result->message, sizeof(result->message), "%s: empty model.", qp ? "QP-IPM" : "IPM");
      return SOV_OK;
    }
    if (f.m <= 0 && !qp) {
      // interior_point.cpp:464-478
      result->status = SOV_OPTIMAL;
      result->has_objective_value = 1;
      double obj = model->obj_constant;
      for (int j = 0; j < f.n_struct; ++j) {
        if (result->primal) result->primal[j] = f.shift[j];
        obj += (model->obj ? model->obj[j] : 0.0) * f.shift[j];
      }
      result->objective_value = obj;
      std::snprintf(result->message, sizeof(result->message), "Optimal (no constraints) via IPM path.");
      return SOV_OK;
    }
    StreamGuard sg;
    sov::solve_single(*model, f, opt, result, sg.s, nullptr);
    return SOV_OK;
  } catch (const sov::CudaError& e) {
    std::snprintf(result->message, sizeof(result->message), "%s error: %s", qp ? "QP-IPM" : "IPM", e.what());
    result->status = SOV_ERROR;
    return set_error(SOV_E_CUDA, e.what());
  } catch (const std::exception& e) {
    std::snprintf(result->message, sizeof(result->message), "%s error: %s", qp ? "QP-IPM" : "IPM", e.what());
    result->status = SOV_ERROR;
    g_last_error = e.what();
    return rc ? rc : SOV_OK;
  }
}

}  // namespace

extern "C" {

void sov_default_lp_options(sov_options* o) {
  std::memset(o, 0, sizeof(*o));
  o->max_iterations = 250;
  o->enable_scaling = 1;
  o->feasibility_tol = 1e-9;
  o->optimality_tol = 1e-9;
  o->fraction_to_boundary = 0.999;
  o->precision = SOV_PRECISION_FP64;
  o->factorization = SOV_FACTOR_AUTO;
  o->pcg_max_iterations = 50;
}

void sov_default_qp_options(sov_options* o) {
  sov_default_lp_options(o);
  o->max_iterations = 100;
  o->enable_scaling = 0;
  o->feasibility_tol = 1e-8;
  o->optimality_tol = 1e-8;
}

int sov_ipm_dims(const sov_model* model, int32_t qp, int32_t* n_ipm, int32_t* m_ipm) {
  int rc = validate(model);
  if (rc) return rc;
  int n_ub = 0, n_slack = 0;
  for (int j = 0; j < model->n; ++j) {
    const double ub = model->ub ? model->ub[j] : 1e30;
    if (std::isfinite(ub) && ub < 1e29) ++n_ub;
  }
  for (int i = 0; i < model->m; ++i) n_slack += model->sense[i] != SOV_EQ ? 1 : 0;
  (void)qp;
  if (n_ipm) *n_ipm = model->n + n_slack + n_ub;
  if (m_ipm) *m_ipm = model->m + n_ub;
  return SOV_OK;
}

int sov_lp_solve(const sov_model* model, const sov_options* opt, sov_result* result) {
  return solve_one(model, opt, result, false);
}

int sov_qp_solve(const sov_model* model, const sov_options* opt, sov_result* result) {
  return solve_one(model, opt, result, true);
}

// Largest bound or row violation of x relative to 1 + |bound| (engine.cpp:60-85); a non-finite
// value counts as infinite.
static double max_relative_violation(const sov_model* p, const double* x) {
  double worst = 0.0;
  std::vector<double> act(p->m, 0.0);
  for (int j = 0; j < p->n; ++j) {
    if (!std::isfinite(x[j])) return INFINITY;
    const double lo = p->lb ? p->lb[j] : 0.0, hi = p->ub ? p->ub[j] : 1e30;
    if (x[j] < lo) worst = std::max(worst, (lo - x[j]) / (1.0 + std::fabs(lo)));
    if (x[j] > hi) worst = std::max(worst, (x[j] - hi) / (1.0 + std::fabs(hi)));
    for (int k = p->col_ptr[j]; k < p->col_ptr[j + 1]; ++k) act[p->row_idx[k]] += p->values[k] * x[j];
  }
  for (int i = 0; i < p->m; ++i) {
    const double v = p->sense[i] == SOV_LE ? act[i] - p->rhs[i]
                     : p->sense[i] == SOV_GE ? p->rhs[i] - act[i]
                                             : std::fabs(act[i] - p->rhs[i]);
    worst = std::max(worst, v / (1.0 + std::fabs(p->rhs[i])));
  }
  return worst;
}

int sov_lp_solve_presolved(const sov_model* model, const sov_options* opt, sov_result* result) {
  if (!result) return set_error(SOV_E_ARGUMENT, "null result");
  reset_result(result);
  int rc = validate(model);
  if (rc) {
    std::snprintf(result->message, sizeof(result->message), "IPM error: %s", g_last_error.c_str());
    return rc;
  }
  sov_presolve* pre = nullptr;
  rc = sov_presolve_lp(model, &pre);
  if (rc) return rc;
  int32_t status = -1;
  sov_presolve_info(pre, &status, nullptr, nullptr, nullptr, nullptr, 0);
  if (status < 0) {
    const sov_model* red = sov_presolve_reduced(pre);
    std::vector<double> x(red->n), dc(red->n), y(red->m);
    sov_result rr = *result;
    rr.primal = x.data();
    rr.dual_col = dc.data();
    rr.dual_row = y.data();
    rr.ipm_x = rr.ipm_y = rr.ipm_s = nullptr;
    rc = solve_one(red, opt, &rr, false);
    if (rc) {
      std::snprintf(result->message, sizeof(result->message), "%s", rr.message);
      sov_presolve_destroy(pre);
      return rc;
    }
    sov_postsolve_lp(pre, &rr, result);
  } else {
    sov_postsolve_lp(pre, nullptr, result);
  }
  sov_presolve_destroy(pre);
  // presolve is checked rather than trusted (engine.cpp:156-176)
  std::string why;
  if (status == SOV_INFEASIBLE) {
    why = std::string("presolve reported infeasibility (") + result->message + ")";
  } else if ((result->status == SOV_OPTIMAL || result->status == SOV_FEASIBLE) && result->primal &&
             max_relative_violation(model, result->primal) > 1e-6) {
    why = "the presolved solution violated the original model";
  }
  if (!why.empty()) {
    rc = solve_one(model, opt, result, false);
    const std::string msg = std::string(result->message) + " | Re-solved without presolve because " + why + ".";
    std::snprintf(result->message, sizeof(result->message), "%s", msg.c_str());
  }
  return rc;
}

int sov_device_info(char* buf, int32_t len) {
  int rc = check_device();
  int dev = 0;
  cudaDeviceProp prop{};
  if (rc == SOV_OK) {
    cudaGetDevice(&dev);
    cudaGetDeviceProperties(&prop, dev);
  }
  if (buf && len > 0) {
    if (rc == SOV_OK)
      std::snprintf(buf, len, "%s (sm_%d%d, %d SMs, %.1f GB HBM, %zu KB smem/block opt-in)", prop.name, prop.major,
                    prop.minor, prop.multiProcessorCount, prop.totalGlobalMem / 1e9, prop.sharedMemPerBlockOptin / 1024);
    else
      std::snprintf(buf, len, "%s", g_last_error.c_str());
  }
  return rc;
}

const char* sov_last_error(void) { return g_last_error.c_str(); }

int sov_spmv_csc(int32_t nrows, int32_t ncols, const int32_t* col_ptr, const int32_t* row_idx, const double* values,
                 const double* x, double* y, int32_t transpose) {
  if (nrows < 0 || ncols < 0 || !col_ptr || !x || !y) return set_error(SOV_E_ARGUMENT, "bad spmv arguments");
  try {
    int rc = check_device();
    if (rc) return rc;
    return sov::spmv_csc_device(nrows, ncols, col_ptr, row_idx, values, x, y, transpose != 0);
  } catch (const std::exception& e) {
    return set_error(SOV_E_CUDA, e.what());
  }
}

int sov_normal_factor_solve(int32_t m, int32_t n, const int32_t* col_ptr, const int32_t* row_idx,
                            const double* values, const double* d, int32_t precision, int32_t factorization,
                            double* rhs, int32_t nrhs, int32_t* dropped_pivots) {
  if (m < 0 || n < 0 || !col_ptr || !d || !rhs || nrhs < 0) return set_error(SOV_E_ARGUMENT, "bad arguments");
  try {
    int rc = check_device();
    if (rc) return rc;
    return sov::normal_factor_solve_device(m, n, col_ptr, row_idx, values, d, precision, factorization, rhs, nrhs,
                                           dropped_pivots);
  } catch (const sov::CudaError& e) {
    return set_error(SOV_E_CUDA, e.what());
  } catch (const std::exception& e) {
    return set_error(SOV_E_ARGUMENT, e.what());
  }
}

int sov_lp_solve_batch(int32_t count, const sov_model* models, const sov_options* opt, int32_t opt_stride,
                       sov_result* results) {
  if (count < 0 || (count > 0 && (!models || !results))) return set_error(SOV_E_ARGUMENT, "bad batch arguments");
  try {
    int rc = check_device();
    if (rc) return rc;
    return sov::solve_batch(count, models, opt, opt_stride, results);
  } catch (const sov::CudaError& e) {
    return set_error(SOV_E_CUDA, e.what());
  } catch (const std::exception& e) {
    return set_error(SOV_E_ARGUMENT, e.what());
  }
}

int sov_lp_solve_family(int32_t count, const sov_model* models, const sov_options* opt, int32_t opt_stride,
                        sov_result* results) {
  if (count < 0 || (count > 0 && (!models || !results))) return set_error(SOV_E_ARGUMENT, "bad family arguments");
  for (int k = 0; k < count; ++k) {
    const int rc = validate(&models[k]);
    if (rc) return rc;
  }
  try {
    int rc = check_device();
    if (rc) return rc;
    return sov::solve_family(count, models, opt, opt_stride, results);
  } catch (const sov::CudaError& e) {
    return set_error(SOV_E_CUDA, e.what());
  } catch (const std::exception& e) {
    return set_error(SOV_E_ARGUMENT, e.what());
  }
}

int sov_batch_create(int32_t count, const sov_model* models, const sov_options* opt, int32_t opt_stride,
                     sov_batch** out) {
  if (count <= 0 || !models || !out) return set_error(SOV_E_ARGUMENT, "bad batch arguments");
  try {
    int rc = check_device();
    if (rc) return rc;
    *out = reinterpret_cast<sov_batch*>(sov::batch_create(count, models, opt, opt_stride));
    return SOV_OK;
  } catch (const sov::CudaError& e) {
    return set_error(SOV_E_CUDA, e.what());
  } catch (const std::exception& e) {
    return set_error(SOV_E_ARGUMENT, e.what());
  }
}

int sov_batch_solve(sov_batch* b, void* stream) {
  if (!b) return set_error(SOV_E_ARGUMENT, "null batch");
  try {
    sov::batch_solve(reinterpret_cast<sov::Batch*>(b), static_cast<cudaStream_t>(stream));
    return SOV_OK;
  } catch (const std::exception& e) {
    return set_error(SOV_E_CUDA, e.what());
  }
}

int sov_batch_results(sov_batch* b, sov_result* results) {
  if (!b || !results) return set_error(SOV_E_ARGUMENT, "null batch or results");
  try {
    sov::batch_results(reinterpret_cast<sov::Batch*>(b), results);
    return SOV_OK;
  } catch (const std::exception& e) {
    return set_error(SOV_E_CUDA, e.what());
  }
}

int sov_batch_stats(const sov_batch* b, int32_t* launches, double* kernel_ms, double* bytes, double* flops) {
  if (!b) return set_error(SOV_E_ARGUMENT, "null batch");
  sov::batch_stats(reinterpret_cast<const sov::Batch*>(b), launches, kernel_ms, bytes, flops);
  return SOV_OK;
}

int sov_batch_transfer_bytes(const sov_batch* b, double* h2d, double* d2h) {
  if (!b) return set_error(SOV_E_ARGUMENT, "null batch");
  sov::batch_transfer_bytes(reinterpret_cast<const sov::Batch*>(b), h2d, d2h);
  return SOV_OK;
}

void sov_batch_destroy(sov_batch* b) { sov::batch_destroy(reinterpret_cast<sov::Batch*>(b)); }

int sov_autotune(int32_t count, const sov_model* models, const sov_options* opt, const char* tuning_file,
                 char* report, int32_t report_len) {
  if (count <= 0 || !models) return set_error(SOV_E_ARGUMENT, "bad autotune arguments");
  try {
    int rc = check_device();
    if (rc) return rc;
    std::string rep = sov::autotune(count, models, opt, tuning_file ? tuning_file : "");
    if (report && report_len > 0) std::snprintf(report, report_len, "%s", rep.c_str());
    return SOV_OK;
  } catch (const std::exception& e) {
    return set_error(SOV_E_CUDA, e.what());
  }
}

}  // extern "C"
