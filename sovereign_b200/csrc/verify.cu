// verify.cu -- certificate of an interior-point answer against the original model, on the GPU.
//
// The primal figures are the checks of the reference's SolutionVerifier::verify
// (solver/core/src/verifier.cpp:10-150): the largest bound violation max(lb - x, x - ub), the largest
// row violation (<=: lhs - rhs, >=: rhs - lhs, =: |lhs - rhs|), the objective recomputed from the
// model (constant + c'x + 1/2 sum of stored q_ij x_i x_j) against the reported one, and the reported
// gap of an OPTIMAL claim. Beside them the dual side that an interior point carries and a vertex
// answer would get from its basis: with the row multipliers y (the published "row_<i>" duals of the
// minimisation form), reduced costs d = c_min + Q x - A'y must be >= 0 on variables with only a lower
// bound, <= 0 with only an upper bound, 0 on free ones; y_i <= 0 on <= rows and >= 0 on >= rows; the
// dual objective b'y - 1/2 x'Qx + sum_j (lb_j max(d_j, 0) + ub_j min(d_j, 0)) is compared with the
// primal one. Activities, objectives and the dual objective are summed in double-double, so the
// figures do not depend on the summation order.
//
// One kernel over rows and columns writes per-block partials; a one-block kernel combines them in
// block order (deterministic).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "dd.cuh"
#include "sov_ipm.h"

namespace sov {
namespace {

constexpr int kCertThreads = 256;
constexpr int kCertBlocks = 148;

struct CertDev {
  int n, m;
  const int *cp, *ri, *rp, *ci, *qp, *qi;  // A by columns and by rows; symmetric Q by columns
  const double *cv, *rv, *qv;
  const double *c, *lb, *ub, *rhs, *x, *y;
  const int8_t* sense;
  double sign;  // +1 minimise, -1 maximise (c_min = sign * c, Q likewise)
};

// per block: max bound viol, max row viol, max reduced-cost sign viol, max row-dual sign viol,
// non-finite count; then dd sums: objective (model sense), b'y, bound terms, x'Qx (min form)
struct Partial {
  double mx[4];
  double nonfinite;
  double sum_hi[4], sum_lo[4];
};

__device__ __forceinline__ dd warp_sum_dd(dd v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const dd w{__shfl_xor_sync(kFull, v.hi, o), __shfl_xor_sync(kFull, v.lo, o)};
    v = dd_add(v, w);
  }
  return v;
}

__global__ void __launch_bounds__(kCertThreads) k_cert_partials(CertDev d, Partial* out) {
  double mx[4] = {0.0, 0.0, 0.0, 0.0};
  double bad = 0.0;
  dd sum[4] = {dd_from(0.0), dd_from(0.0), dd_from(0.0), dd_from(0.0)};
  const int total = d.n + d.m;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    if (t < d.n) {
      const int j = t;
      const double xj = d.x[j];
      if (!isfinite(xj)) {
        bad += 1.0;
        continue;
      }
      const double lo = d.lb ? d.lb[j] : 0.0, hi = d.ub ? d.ub[j] : 1e30;
      mx[0] = fmax(mx[0], fmax(lo - xj, xj - hi));
      dd qx = dd_from(0.0);  // (Q x)_j of the model's Q (symmetric form)
      if (d.qp)
        for (int e = d.qp[j]; e < d.qp[j + 1]; ++e) qx = dd_add(qx, two_prod(d.qv[e], d.x[d.qi[e]]));
      const double cj = d.c ? d.c[j] : 0.0;
      // objective in the model's sense: c_j x_j + 1/2 x_j (Qx)_j
      sum[0] = dd_add(sum[0], dd_add(two_prod(cj, xj), dd_mul_d(qx, 0.5 * xj)));
      sum[3] = dd_add(sum[3], dd_mul_d(qx, d.sign * xj));  // x'Qx of the minimisation form
      dd aty = dd_from(0.0);
      for (int e = d.cp[j]; e < d.cp[j + 1]; ++e) aty = dd_add(aty, two_prod(d.cv[e], d.y[d.ri[e]]));
      const double dj = dd_sub(dd_add(dd_from(d.sign * cj), dd_mul_d(qx, d.sign)), aty).hi;
      const bool has_lo = lo > -1e29, has_hi = hi < 1e29;
      if (has_lo && has_hi) {
        sum[2] = dd_add(sum[2], two_prod(dj > 0.0 ? lo : hi, dj));
      } else if (has_lo) {
        mx[2] = fmax(mx[2], -dj);
        sum[2] = dd_add(sum[2], two_prod(lo, fmax(dj, 0.0)));
      } else if (has_hi) {
        mx[2] = fmax(mx[2], dj);
        sum[2] = dd_add(sum[2], two_prod(hi, fmin(dj, 0.0)));
      } else {
        mx[2] = fmax(mx[2], fabs(dj));
      }
    } else {
      const int i = t - d.n;
      dd lhs = dd_from(0.0);
      for (int e = d.rp[i]; e < d.rp[i + 1]; ++e) lhs = dd_add(lhs, two_prod(d.rv[e], d.x[d.ci[e]]));
      const double act = lhs.hi + lhs.lo;
      if (!isfinite(act)) {
        bad += 1.0;
        continue;
      }
      const double b = d.rhs[i], yi = d.y[i];
      const int s = d.sense[i];
      mx[1] = fmax(mx[1], s == SOV_LE ? act - b : s == SOV_GE ? b - act : fabs(act - b));
      if (s == SOV_LE) mx[3] = fmax(mx[3], yi);
      if (s == SOV_GE) mx[3] = fmax(mx[3], -yi);
      sum[1] = dd_add(sum[1], two_prod(b, yi));
    }
  }
  __shared__ double smx[5][kCertThreads / 32];
  __shared__ double shi[4][kCertThreads / 32], slo[4][kCertThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const double w = warp_max(mx[k]);
    const dd sv = warp_sum_dd(sum[k]);
    if (lane == 0) {
      smx[k][warp] = w;
      shi[k][warp] = sv.hi;
      slo[k][warp] = sv.lo;
    }
  }
  const double bw = warp_sum(bad);
  if (lane == 0) smx[4][warp] = bw;
  __syncthreads();
  if (threadIdx.x == 0) {
    Partial p;
    for (int k = 0; k < 4; ++k) {
      p.mx[k] = 0.0;
      dd s = dd_from(0.0);
      for (int w = 0; w < kCertThreads / 32; ++w) {
        p.mx[k] = fmax(p.mx[k], smx[k][w]);
        s = dd_add(s, dd{shi[k][w], slo[k][w]});
      }
      p.sum_hi[k] = s.hi;
      p.sum_lo[k] = s.lo;
    }
    p.nonfinite = 0.0;
    for (int w = 0; w < kCertThreads / 32; ++w) p.nonfinite += smx[4][w];
    out[blockIdx.x] = p;
  }
}

__global__ void k_cert_final(const Partial* parts, int count, Partial* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  Partial r;
  for (int k = 0; k < 4; ++k) {
    r.mx[k] = 0.0;
    dd s = dd_from(0.0);
    for (int b = 0; b < count; ++b) {
      r.mx[k] = fmax(r.mx[k], parts[b].mx[k]);
      s = dd_add(s, dd{parts[b].sum_hi[k], parts[b].sum_lo[k]});
    }
    r.sum_hi[k] = s.hi;
    r.sum_lo[k] = s.lo;
  }
  r.nonfinite = 0.0;
  for (int b = 0; b < count; ++b) r.nonfinite += parts[b].nonfinite;
  *out = r;
}

template <class T>
struct CertBuf {
  T* p = nullptr;
  explicit CertBuf(size_t count) { SOV_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(count, 1))); }
  ~CertBuf() {
    if (p) cudaFree(p);
  }
  CertBuf(const CertBuf&) = delete;
  CertBuf& operator=(const CertBuf&) = delete;
};

template <class T>
T* upload(CertBuf<T>& b, const T* h, size_t count) {
  if (count) SOV_CUDA(cudaMemcpy(b.p, h, sizeof(T) * count, cudaMemcpyHostToDevice));
  return b.p;
}

}  // namespace
}  // namespace sov

extern "C" int sov_verify_solution(const sov_model* p, const sov_result* res, double tol, sov_certificate* cert) {
  using namespace sov;
  if (!p || !res || !cert || p->n < 0 || p->m < 0 || !(tol >= 0.0))
    return record_error(SOV_E_ARGUMENT, "verify: null argument, negative size or bad tolerance");
  if (p->n > 0 && (!p->col_ptr || !res->primal)) return record_error(SOV_E_ARGUMENT, "verify: missing primal or A");
  if (p->m > 0 && (!p->sense || !p->rhs || !res->dual_row))
    return record_error(SOV_E_ARGUMENT, "verify: missing row data or row duals");
  const int nnz = p->n > 0 ? p->col_ptr[p->n] : 0;
  for (int j = 0; j < p->n; ++j)
    if (p->col_ptr[j + 1] < p->col_ptr[j]) return record_error(SOV_E_ARGUMENT, "verify: col_ptr is not monotone");
  for (int k = 0; k < nnz; ++k)
    if (p->row_idx[k] < 0 || p->row_idx[k] >= p->m) return record_error(SOV_E_ARGUMENT, "verify: row index out of range");
  if (int rc = require_device()) return rc;
  std::memset(cert, 0, sizeof(*cert));
  try {
    const int n = p->n, m = p->m;
    // rows of A (the activity of each row) and the symmetric form of the stored Q terms
    std::vector<int> rp(m + 1, 0), ci(nnz);
    std::vector<double> rv(nnz);
    for (int k = 0; k < nnz; ++k) rp[p->row_idx[k] + 1]++;
    for (int i = 0; i < m; ++i) rp[i + 1] += rp[i];
    {
      std::vector<int> at(rp.begin(), rp.end() - 1);
      for (int j = 0; j < n; ++j)
        for (int k = p->col_ptr[j]; k < p->col_ptr[j + 1]; ++k) {
          ci[at[p->row_idx[k]]] = j;
          rv[at[p->row_idx[k]]++] = p->values[k];
        }
    }
    std::vector<int> qp, qi;
    std::vector<double> qv;
    if (p->q_col_ptr) {  // gradient of 1/2 sum q_ij x_i x_j: (q_ij / 2) x_j to i and (q_ij / 2) x_i to j
      std::vector<std::vector<std::pair<int, double>>> cols(n);
      for (int j = 0; j < n; ++j)
        for (int k = p->q_col_ptr[j]; k < p->q_col_ptr[j + 1]; ++k) {
          const int i = p->q_row_idx[k];
          if (i < 0 || i >= n) return record_error(SOV_E_ARGUMENT, "verify: Q row index out of range");
          cols[j].push_back({i, 0.5 * p->q_values[k]});
          cols[i].push_back({j, 0.5 * p->q_values[k]});
        }
      qp.assign(n + 1, 0);
      for (int j = 0; j < n; ++j) {
        for (const auto& e : cols[j]) {
          qi.push_back(e.first);
          qv.push_back(e.second);
        }
        qp[j + 1] = static_cast<int>(qi.size());
      }
    }
    CertBuf<int> d_cp(n + 1), d_ri(nnz), d_rp(m + 1), d_ci(nnz), d_qp(qp.size()), d_qi(qi.size());
    CertBuf<double> d_cv(nnz), d_rv(nnz), d_qv(qv.size()), d_c(n), d_lb(n), d_ub(n), d_rhs(m), d_x(n), d_y(m);
    CertBuf<int8_t> d_sense(m);
    CertBuf<Partial> d_parts(kCertBlocks), d_out(1);
    CertDev d{};
    d.n = n;
    d.m = m;
    d.cp = upload(d_cp, p->col_ptr, n + 1);
    d.ri = upload(d_ri, p->row_idx, nnz);
    d.cv = upload(d_cv, p->values, nnz);
    d.rp = upload(d_rp, rp.data(), m + 1);
    d.ci = upload(d_ci, ci.data(), nnz);
    d.rv = upload(d_rv, rv.data(), nnz);
    if (!qp.empty()) {
      d.qp = upload(d_qp, qp.data(), qp.size());
      d.qi = upload(d_qi, qi.data(), qi.size());
      d.qv = upload(d_qv, qv.data(), qv.size());
    }
    d.c = p->obj ? upload(d_c, p->obj, n) : nullptr;
    d.lb = p->lb ? upload(d_lb, p->lb, n) : nullptr;
    d.ub = p->ub ? upload(d_ub, p->ub, n) : nullptr;
    d.rhs = upload(d_rhs, p->rhs, m);
    d.sense = upload(d_sense, p->sense, m);
    d.x = upload(d_x, res->primal, n);
    d.y = upload(d_y, res->dual_row, m);
    d.sign = p->maximize ? -1.0 : 1.0;
    k_cert_partials<<<kCertBlocks, kCertThreads>>>(d, d_parts.p);
    k_cert_final<<<1, 32>>>(d_parts.p, kCertBlocks, d_out.p);
    SOV_LAUNCH_CHECK();
    Partial r;
    SOV_CUDA(cudaMemcpy(&r, d_out.p, sizeof(Partial), cudaMemcpyDeviceToHost));
    const double obj = r.sum_hi[0] + r.sum_lo[0] + p->obj_constant;
    const double xqx = r.sum_hi[3] + r.sum_lo[3];
    const double primal_min = p->maximize ? -obj : obj;
    const double dual_min = (r.sum_hi[1] + r.sum_lo[1]) + (r.sum_hi[2] + r.sum_lo[2]) - 0.5 * xqx +
                            (p->maximize ? -p->obj_constant : p->obj_constant);
    cert->max_bound_violation = r.mx[0];
    cert->max_constraint_violation = r.mx[1];
    cert->max_dual_infeasibility = std::max(r.mx[2], r.mx[3]);
    cert->recomputed_objective = obj;
    cert->dual_objective = p->maximize ? -dual_min : dual_min;
    cert->relative_gap = std::fabs(primal_min - dual_min) / (1.0 + std::fabs(primal_min));
    cert->nonfinite = static_cast<int32_t>(r.nonfinite);
    // the verifier's verdict (verifier.cpp:17-38, 100-148)
    int issues = 0;
    const int st = res->status;
    if (st == SOV_NOT_IMPLEMENTED || st == SOV_ERROR || st == SOV_NUMERICAL_ERROR || st == SOV_TIME_LIMIT ||
        st == SOV_ITERATION_LIMIT)
      issues |= SOV_CERT_NO_FEASIBLE_STATUS;
    else if (st == SOV_INFEASIBLE || st == SOV_UNBOUNDED)
      issues |= SOV_CERT_UNCHECKABLE_STATUS;
    else {
      if (cert->nonfinite) issues |= SOV_CERT_NONFINITE;
      if (cert->max_bound_violation > tol) issues |= SOV_CERT_BOUND;
      if (cert->max_constraint_violation > tol) issues |= SOV_CERT_CONSTRAINT;
      if (res->has_objective_value && std::fabs(res->objective_value - obj) > tol * (1.0 + std::fabs(obj)))
        issues |= SOV_CERT_OBJECTIVE;
      if (st == SOV_OPTIMAL && res->duality_gap > tol) issues |= SOV_CERT_GAP;
    }
    cert->issues = issues;
    cert->is_valid = issues == 0 ? 1 : 0;
    return SOV_OK;
  } catch (const std::exception& e) {
    return record_error(SOV_E_CUDA, std::string("verify: ") + e.what());
  }
}
