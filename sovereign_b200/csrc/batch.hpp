// batch.hpp -- batched persistent interior-point solver (one CTA per LP) and device tools.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "sov_ipm.h"

namespace sov {

struct Batch;

// Starts already on the device for every LP of a call (a warm-start network's output): LP k's
// x at x + k*n, y at y + k*m, s at s + k*n; every batched LP must have n IPM columns and m rows.
struct DeviceStarts {
  const double *x, *y, *s;
  int n, m;
  cudaEvent_t ready;  // recorded when the starts are written (or null: already written)
};

int solve_batch(int count, const sov_model* models, const sov_options* opt, int opt_stride, sov_result* results,
                const DeviceStarts* starts = nullptr);
// first_lp: the caller's position of models[0] (a part of a larger call), for the device starts
// and the model numbers in errors
Batch* batch_create(int count, const sov_model* models, const sov_options* opt, int opt_stride = 0,
                    const DeviceStarts* starts = nullptr, int first_lp = 0);
void batch_solve(Batch* b, cudaStream_t st);
void batch_results(Batch* b, sov_result* results);
void batch_stats(const Batch* b, int* launches, double* kernel_ms, double* bytes, double* flops);
void batch_transfer_bytes(const Batch* b, double* h2d, double* d2h);
void batch_destroy(Batch* b);
std::string autotune(int count, const sov_model* models, const sov_options* opt, const std::string& file);
// memcpy of a large host range on the library's worker threads (chunks of 256 KB)
void parallel_memcpy(void* dst, const void* src, size_t bytes);

// y = A x / A' x for a host CSC matrix (device kernels; host buffers in and out)
int spmv_csc_device(int nrows, int ncols, const int* col_ptr, const int* row_idx, const double* values,
                    const double* x, double* y, bool transpose);
// factor A diag(d) A' + 1e-12 I and solve for nrhs right-hand sides (host buffers)
int normal_factor_solve_device(int m, int n, const int* col_ptr, const int* row_idx, const double* values,
                               const double* d, int precision, int factorization, double* rhs, int nrhs,
                               int* dropped);

}  // namespace sov
