// tools.cu -- stand-alone device entry points for the kernels the IPM is built from.
//
// sov_spmv_csc mirrors spmv_csc_auto (solver/gpu/src/gpu_spmv.cpp:70-102): y = A x sums each
// row's terms in column order and y = A' x each column's terms in row order, the orders of the
// reference's CPU loops (gpu_spmv.cpp:42-50, 58-66), with separately rounded multiply and add so
// the result is bit-identical to the reference's.
// sov_normal_factor_solve runs the normal-equation backends on one system.
#include <algorithm>
#include <cmath>
#include <vector>

#include "band.cuh"
#include "batch.hpp"
#include "common.cuh"
#include "dense.cuh"
#include "stdform.hpp"

namespace sov {
namespace {

__global__ void k_spmv_rows_exact(int m, const int* __restrict__ rp, const int* __restrict__ ci,
                                  const double* __restrict__ v, const double* __restrict__ x, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double acc = 0.0;
  for (int p = rp[i]; p < rp[i + 1]; ++p) {
    const double xj = x[ci[p]];
    if (xj == 0.0) continue;  // the reference skips zero x_j (gpu_spmv.cpp:45)
    acc = __dadd_rn(acc, __dmul_rn(v[p], xj));
  }
  y[i] = acc;
}

__global__ void k_spmv_cols_exact(int n, const int* __restrict__ cp, const int* __restrict__ ri,
                                  const double* __restrict__ v, const double* __restrict__ x, double* __restrict__ y) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  double acc = 0.0;
  for (int p = cp[j]; p < cp[j + 1]; ++p) acc = __dadd_rn(acc, __dmul_rn(v[p], x[ri[p]]));
  y[j] = acc;
}

template <class T>
struct Tmp {
  T* p = nullptr;
  explicit Tmp(size_t n) {
    if (n) SOV_CUDA(cudaMalloc(&p, sizeof(T) * n));
  }
  void put(const T* h, size_t n) {
    if (n) SOV_CUDA(cudaMemcpy(p, h, sizeof(T) * n, cudaMemcpyHostToDevice));
  }
  void get(T* h, size_t n) const {
    if (n) SOV_CUDA(cudaMemcpy(h, p, sizeof(T) * n, cudaMemcpyDeviceToHost));
  }
  ~Tmp() {
    if (p) cudaFree(p);
  }
};

}  // namespace

int spmv_csc_device(int nrows, int ncols, const int* col_ptr, const int* row_idx, const double* values,
                    const double* x, double* y, bool transpose) {
  const int nnz = ncols > 0 ? col_ptr[ncols] : 0;
  if (!transpose) {
    // rows of A in column order = CSR with sorted columns
    std::vector<int> rp(nrows + 1, 0), ci(nnz);
    std::vector<double> rv(nnz);
    for (int k = 0; k < nnz; ++k) rp[row_idx[k] + 1]++;
    for (int i = 0; i < nrows; ++i) rp[i + 1] += rp[i];
    std::vector<int> fill(rp.begin(), rp.end() - 1);
    for (int j = 0; j < ncols; ++j)
      for (int k = col_ptr[j]; k < col_ptr[j + 1]; ++k) {
        const int q = fill[row_idx[k]]++;
        ci[q] = j;
        rv[q] = values[k];
      }
    Tmp<int> drp(nrows + 1), dci(nnz);
    Tmp<double> drv(nnz), dx(ncols), dy(nrows);
    drp.put(rp.data(), nrows + 1);
    dci.put(ci.data(), nnz);
    drv.put(rv.data(), nnz);
    dx.put(x, ncols);
    if (nrows) k_spmv_rows_exact<<<ceil_div(nrows, 256), 256>>>(nrows, drp.p, dci.p, drv.p, dx.p, dy.p);
    SOV_LAUNCH_CHECK();
    dy.get(y, nrows);
  } else {
    Tmp<int> dcp(ncols + 1), dri(nnz);
    Tmp<double> dv(nnz), dx(nrows), dy(ncols);
    dcp.put(col_ptr, ncols + 1);
    dri.put(row_idx, nnz);
    dv.put(values, nnz);
    dx.put(x, nrows);
    if (ncols) k_spmv_cols_exact<<<ceil_div(ncols, 256), 256>>>(ncols, dcp.p, dri.p, dv.p, dx.p, dy.p);
    SOV_LAUNCH_CHECK();
    dy.get(y, ncols);
  }
  SOV_CUDA(cudaDeviceSynchronize());
  return SOV_OK;
}

int normal_factor_solve_device(int m, int n, const int* col_ptr, const int* row_idx, const double* values,
                               const double* d, int precision, int factorization, double* rhs, int nrhs,
                               int* dropped) {
  StdForm f;
  f.m = m;
  f.n = n;
  f.col_ptr.assign(col_ptr, col_ptr + n + 1);
  const int nnz = col_ptr[n];
  f.row_idx.assign(row_idx, row_idx + nnz);
  f.val.assign(values, values + nnz);
  // the kernels compute the column weight as max(x,1e-16)/max(s,1e-16); pass x = d, s = 1
  std::vector<double> ones(n, 1.0);
  Tmp<double> dx(n), ds(n), ddiag(m);
  dx.put(d, n);
  ds.put(ones.data(), n);
  Tmp<int> counters(3);
  SOV_CUDA(cudaMemset(counters.p, 0, 2 * sizeof(int)));
  const int kd = normal_bandwidth(f);
  const bool band = factorization == SOV_FACTOR_BANDED || (factorization == SOV_FACTOR_AUTO && kd <= kBandMax && m > 256);
  auto upload_map = [&](const AssemblyMap& am, Tmp<int64_t>& t, Tmp<int>& ptr, Tmp<int>& col, Tmp<double>& w) {
    t.put(am.target.data(), am.target.size());
    ptr.put(am.ptr.data(), am.ptr.size());
    col.put(am.col.data(), am.col.size());
    w.put(am.w.data(), am.w.size());
  };
  int drops = 0;
  if (band) {
    if (kd > kBandMax) throw std::runtime_error("half-bandwidth exceeds the band kernels' limit");
    AssemblyMap am = build_assembly_band(f, kd);
    Tmp<int64_t> t(am.target.size());
    Tmp<int> ptr(am.ptr.size()), col(am.col.size());
    Tmp<double> w(am.w.size());
    upload_map(am, t, ptr, col, w);
    Tmp<double> B(static_cast<size_t>(kBandMax + 1) * m), dinv(m), z(m);
    SOV_CUDA(cudaMemset(B.p, 0, sizeof(double) * (kBandMax + 1) * m));
    AssemblyDev ad{t.p, ptr.p, col.p, w.p, nullptr, static_cast<int>(am.target.size())};
    launch_assemble<double>(ad, dx.p, ds.p, nullptr, nullptr, kWeightLp, 1e-12, B.p, ddiag.p, m, -m, 0);
    BandSystem bs{B.p, dinv.p, ddiag.p, m, kd, counters.p, counters.p + 1};
    band_factor(bs, 0, nullptr);
    for (int r = 0; r < nrhs; ++r) {
      z.put(rhs + static_cast<size_t>(r) * m, m);
      band_solve(bs, z.p, 0, nullptr);
      z.get(rhs + static_cast<size_t>(r) * m, m);
    }
  } else {
    const int nb = ceil_div(m, kNB), mp = nb * kNB;
    AssemblyMap am = build_assembly_dense(f, mp);
    Tmp<int64_t> t(am.target.size());
    Tmp<int> ptr(am.ptr.size()), col(am.col.size());
    Tmp<double> w(am.w.size());
    upload_map(am, t, ptr, col, w);
    AssemblyDev ad{t.p, ptr.p, col.p, w.p, nullptr, static_cast<int>(am.target.size())};
    Tmp<unsigned> flags(nb);
    SOV_CUDA(cudaMemset(flags.p, 0, sizeof(unsigned) * nb));
    Tmp<int> err(1);
    SOV_CUDA(cudaMemset(err.p, 0, sizeof(int)));
    Tmp<double> z(mp);
    SOV_CUDA(cudaMemset(z.p, 0, sizeof(double) * mp));
    unsigned epoch = 0;
    if (precision == SOV_PRECISION_FP64) {
      Tmp<double> M(static_cast<size_t>(mp) * mp), Linv(static_cast<size_t>(nb) * kNB * kNB);
      launch_dense_clear<double>(M.p, m, mp, 0);
      launch_assemble<double>(ad, dx.p, ds.p, nullptr, nullptr, kWeightLp, 1e-12, M.p, ddiag.p, m, mp, 0);
      DenseSystem<double> s{M.p, Linv.p, ddiag.p, m, mp, nb, counters.p, counters.p + 1, flags.p,
                                reinterpret_cast<unsigned*>(counters.p + 2), 1e-13};
      dense_cholesky<double>(s, 0, nullptr);
      for (int r = 0; r < nrhs; ++r) {
        z.put(rhs + static_cast<size_t>(r) * m, m);
        dense_solve<double>(s, z.p, epoch, err.p, 0, nullptr);
        z.get(rhs + static_cast<size_t>(r) * m, m);
      }
    } else {
      Tmp<float> M(static_cast<size_t>(mp) * mp), Linv(static_cast<size_t>(nb) * kNB * kNB);
      launch_dense_clear<float>(M.p, m, mp, 0);
      launch_assemble<float>(ad, dx.p, ds.p, nullptr, nullptr, kWeightLp, 1e-12, M.p, ddiag.p, m, mp, 0);
      DenseSystem<float> s{M.p, Linv.p, ddiag.p, m, mp, nb, counters.p, counters.p + 1, flags.p,
                               reinterpret_cast<unsigned*>(counters.p + 2), 1e-6};
      dense_cholesky_tc(s, err.p, 0, nullptr);
      for (int r = 0; r < nrhs; ++r) {
        z.put(rhs + static_cast<size_t>(r) * m, m);
        dense_solve<float>(s, z.p, epoch, err.p, 0, nullptr);
        z.get(rhs + static_cast<size_t>(r) * m, m);
      }
    }
    int e = 0;
    err.get(&e, 1);
    if (e) throw CudaError("dataflow triangular solve timed out");
  }
  int h[2] = {0, 0};
  counters.get(h, 2);
  drops = h[0];
  if (dropped) *dropped = drops;
  SOV_CUDA(cudaDeviceSynchronize());
  return h[1] ? SOV_E_CUDA : SOV_OK;
}

}  // namespace sov
