// ipm_kernels.cu -- per-iteration vector kernels of the Mehrotra predictor-corrector method.
//
// Every pass is fused so that each n- or m-vector crosses HBM once per logical use:
//   residual rows    rp = b - A x                               + max|rp|
//   residual cols    rd = c + Qx - A'y - s                      + max|rd|, x's, c'x, x'Qx
//   Newton rhs rows  z = rp + A tmp, tmp from (x, s, rd, dx_aff, ds_aff, sigma mu) on the fly
//   direction cols   A'dy, dx, ds, both ratio tests             (+ mu_aff pass for the predictor)
//   update           x, s (floors) and y
// Reductions are deterministic: per-block partials, the last block to finish folds them in
// block order and applies the scalar logic of the reference (mu, residual norms, gap, sigma,
// step lengths), so the host reads one small struct per iteration.
#include <algorithm>

#include "common.cuh"
#include "ipm_kernels.cuh"

namespace sov {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1184;  // 8 x 148 SMs

__device__ __forceinline__ double op_apply(int op, double a, double b) {
  return op == 0 ? a + b : op == 1 ? fmax(a, b) : fmin(a, b);
}
__device__ __forceinline__ double op_identity(int op) { return op == 0 ? 0.0 : op == 1 ? -INFINITY : INFINITY; }

// Block-reduce NV values, publish partials, and return true in every thread of the last block,
// whose thread 0 then holds the grid-wide results in v.
template <int NV>
__device__ bool grid_reduce(double (&v)[NV], const int (&ops)[NV], double* partials, unsigned* counter) {
  __shared__ double scratch[4 * 32];
  __shared__ bool last;
  static_assert(NV <= 8, "at most 8 slots");
  // reduce in chunks of 4 through the shared scratch
  double r[NV];
#pragma unroll
  for (int k0 = 0; k0 < NV; k0 += 4) {
    double t[4];
    int o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      t[k] = k0 + k < NV ? v[k0 + k] : 0.0;
      o[k] = k0 + k < NV ? ops[k0 + k] : 0;
    }
    block_reduce<4>(t, o, scratch);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k0 + k < NV) r[k0 + k] = t[k];
  }
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[k * kMaxBlocks + blockIdx.x] = r[k];
    __threadfence();
    const unsigned ticket = atomicAdd(counter, 1u);
    last = ticket == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
#pragma unroll
  for (int k0 = 0; k0 < NV; k0 += 4) {
    double t[4];
    int o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      o[k] = k0 + k < NV ? ops[k0 + k] : 0;
      double acc = op_identity(o[k]);
      if (k0 + k < NV)
        for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
          acc = op_apply(o[k], acc, __ldcg(partials + (k0 + k) * kMaxBlocks + b));
      t[k] = acc;
    }
    block_reduce<4>(t, o, scratch);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k0 + k < NV) v[k0 + k] = t[k];
  }
  if (threadIdx.x == 0) *counter = 0;
  return true;
}

int blocks_for(int n) { return std::max(1, std::min(kMaxBlocks, ceil_div(n, kThreads))); }

// sum_j a_ij v_j over row i, one warp per row
__device__ __forceinline__ int warp_row() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }

// sum over p = first, first + stride, ... < end of term(p), accumulated in that order, four terms'
// loads issued before their products are added (the dependent gathers of several entries overlap)
template <class Term>
__device__ __forceinline__ double strided_sum(int first, int end, int stride, Term term) {
  double acc = 0.0;
  int p = first;
  for (; p + 3 * stride < end; p += 4 * stride) {
    const double t0 = term(p), t1 = term(p + stride), t2 = term(p + 2 * stride), t3 = term(p + 3 * stride);
    acc += t0;
    acc += t1;
    acc += t2;
    acc += t3;
  }
  for (; p < end; p += stride) acc += term(p);
  return acc;
}

// sum_p a_pj v[row_p] over column j, in entry order
__device__ __forceinline__ double col_dot(const IpmDev& d, int j, const double* v) {
  return strided_sum(d.col_ptr[j], d.col_ptr[j + 1], 1, [&](int p) { return d.cval[p] * v[d.row_idx[p]]; });
}

// Row sums sum_p term(p) over the entries of each row, handed to out(i, sum) on one thread: a warp
// per row; for long rows on average (d.row_block), the whole CTA per row so that enough loads are
// in flight to stream A from HBM; when some row is longer than a piece (d.row_piece: a dense row),
// a warp per piece -- rows cut into pieces leave their piece sums in d.row_partial for the
// kernel's combine launch (for_each_cut_row). Partial sums are added in a fixed order throughout.
template <class Term, class Out>
__device__ __forceinline__ void for_each_row(const IpmDev& d, Term term, Out out) {
  if (d.row_piece) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (blockDim.x >> 5);
    for (int q = warp_row(); q < d.row_pieces; q += warps) {
      const int4 pc = d.row_piece[q];
      double acc = strided_sum(pc.x + lane, pc.y, 32, term);
      acc = warp_sum(acc);
      if (lane == 0) {
        if (pc.w < 0) out(pc.z, acc);
        else d.row_partial[pc.w] = acc;
      }
    }
    return;
  }
  if (d.row_block) {
    __shared__ double part[kThreads / 32];
    for (int i = blockIdx.x; i < d.m; i += gridDim.x) {  // uniform over the CTA: barriers are safe
      double acc = strided_sum(d.row_ptr[i] + threadIdx.x, d.row_ptr[i + 1], blockDim.x, term);
      acc = warp_sum(acc);
      if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
      __syncthreads();
      if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += part[w];
        out(i, t);
      }
      __syncthreads();
    }
    return;
  }
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = warp_row(); i < d.m; i += warps) {
    double acc = strided_sum(d.row_ptr[i] + lane, d.row_ptr[i + 1], 32, term);
    acc = warp_sum(acc);
    if (lane == 0) out(i, acc);
  }
}

// ---------------------------------------------------------------------------------------------
// The rows that for_each_row cut into pieces: their piece sums added in order, handed to out.
template <class Out>
__device__ __forceinline__ void for_each_cut_row(const IpmDev& d, Out out) {
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.row_combs; c += gridDim.x * blockDim.x) {
    const int4 cb = d.row_comb[c];
    double acc = 0.0;
    for (int k = 0; k < cb.z; ++k) acc += d.row_partial[cb.y + k];
    out(cb.x, acc);
  }
}

__global__ void __launch_bounds__(kThreads) k_residual_rows(IpmDev d) {
  double mx = 0.0;
  for_each_row(
      d, [&](int p) { return d.rval[p] * d.x[d.col_idx[p]]; },
      [&](int i, double acc) {
        const double r = d.b[i] - acc;
        d.rp[i] = r;
        mx = fmax(mx, fabs(r));
      });
  double v[1] = {mx};
  const int ops[1] = {1};
  if (grid_reduce<1>(v, ops, d.partials, d.counter) && threadIdx.x == 0) d.sc->rp_max = v[0];
}

// one CTA: the cut rows' residuals, and their maximum folded into sc->rp_max
__global__ void __launch_bounds__(kThreads) k_residual_rows_cut(IpmDev d) {
  __shared__ double red[4 * 32];
  double mx = 0.0;
  for_each_cut_row(d, [&](int i, double acc) {
    const double r = d.b[i] - acc;
    d.rp[i] = r;
    mx = fmax(mx, fabs(r));
  });
  double v[1] = {mx};
  const int ops[1] = {1};
  block_reduce<1>(v, ops, red);
  if (threadIdx.x == 0) d.sc->rp_max = fmax(d.sc->rp_max, v[0]);
}

__global__ void __launch_bounds__(kThreads) k_residual_cols(IpmDev d) {
  double rdm = 0.0, xs = 0.0, cx = 0.0, xqx = 0.0, qxm = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    const double aty = col_dot(d, j, d.y);
    const double xj = d.x[j], sj = d.s[j];
    double qx = 0.0;
    if (d.qp) {
      if (d.q_coupled) {  // (Q x)_j from column j of the symmetric Q
        for (int k = d.q_ptr[j]; k < d.q_ptr[j + 1]; ++k) qx += d.q_val[k] * d.x[d.q_idx[k]];
      } else {
        qx = d.qdiag[j] * xj;
      }
    }
    // LP: rd = c - (A'y + s) (interior_point.cpp:578-582); QP: Qx + c - A'y - s (:2986-2992)
    const double r = d.qp ? qx + d.c[j] - aty - sj : d.c[j] - (aty + sj);
    d.rd[j] = r;
    rdm = fmax(rdm, fabs(r));
    if (!d.qp || !d.free_col[j]) xs += xj * sj;
    cx += d.c[j] * xj;
    xqx += xj * qx;
    qxm = fmax(qxm, fabs(qx));
  }
  double v[5] = {rdm, xs, cx, xqx, qxm};
  const int ops[5] = {1, 0, 0, 0, 1};
  if (grid_reduce<5>(v, ops, d.partials, d.counter) && threadIdx.x == 0) {
    IpmScalars* sc = d.sc;
    sc->rd_max = v[0];
    sc->xs = v[1];
    sc->cx = v[2];
    sc->xqx = v[3];
    sc->qx_max = v[4];
    sc->p_res = sc->rp_max / d.bnorm;
    if (d.qp) {
      sc->mu = v[1] / d.comp_count;
      sc->d_res = v[0] / fmax(1.0, d.cnorm + v[4]);
      sc->gap = sc->mu * d.comp_count / (1.0 + fabs(v[2] + 0.5 * v[3] + d.objective_offset));
    } else {
      sc->mu = v[1] / static_cast<double>(d.n);
      sc->d_res = v[0] / d.cnorm;
      sc->gap = fabs(v[1]) / (1.0 + fabs(v[2]));
    }
    sc->metric = fmax(sc->p_res, fmax(sc->d_res, sc->gap));
  }
}

// Complementarity right-hand side rxs_j of the current mode (interior_point.cpp:644-648,
// 676-681; qp_interior_point.cpp:3051-3055, 3075-3080).
__device__ __forceinline__ double rxs_of(const IpmDev& d, int mode, int j, double sigma_mu) {
  const double xj = d.x[j], sj = d.s[j];
  if (d.qp && d.free_col[j]) return 0.0;
  if (mode == kRhsAffine) return -xj * sj;
  return -xj * sj - d.dxa[j] * d.dsa[j] + sigma_mu;
}

// tmp_j of z = rp + A tmp:  LP: d rd - rxs/s ; QP: -D r1 with D = 1/(Q_jj + h), r1 = -rd + rxs/x
__device__ __forceinline__ double newton_tmp(const IpmDev& d, int mode, int j, double sigma_mu) {
  const double xj = fmax(d.x[j], 1e-16), sj = fmax(d.s[j], 1e-16);
  const double rxs = rxs_of(d, mode, j, sigma_mu);
  if (!d.qp) return (xj / sj) * d.rd[j] - rxs / sj;
  const bool fr = d.free_col[j];
  const double D = 1.0 / (d.qdiag[j] + (fr ? 0.0 : sj / xj));
  const double r1 = fr ? -d.rd[j] : -d.rd[j] + rxs / xj;
  return -D * r1;
}

__global__ void __launch_bounds__(kThreads) k_newton_rhs(IpmDev d, int mode) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  auto out = [&](int i, double acc) { d.z[i] = d.rp[i] + acc; };
  if (d.coltmp)  // tmp_j computed once per column by k_newton_tmp
    for_each_row(d, [&](int p) { return d.rval[p] * d.coltmp[d.col_idx[p]]; }, out);
  else
    for_each_row(d, [&](int p) { return d.rval[p] * newton_tmp(d, mode, d.col_idx[p], sigma_mu); }, out);
}

__global__ void __launch_bounds__(kThreads) k_newton_rhs_cut(IpmDev d) {
  for_each_cut_row(d, [&](int i, double acc) { d.z[i] = d.rp[i] + acc; });
}

__global__ void __launch_bounds__(kThreads) k_newton_tmp(IpmDev d, int mode) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x)
    d.coltmp[j] = newton_tmp(d, mode, j, sigma_mu);
}

__global__ void __launch_bounds__(kThreads) k_direction(IpmDev d, int mode, const double* dxv) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  double* dx = mode == kRhsAffine ? d.dxa : d.dx;
  double* ds = mode == kRhsAffine ? d.dsa : d.ds;
  double rp_min = 1.0, rd_min = 1.0;  // step_to_bound starts at alpha = 1
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    const double atdy = col_dot(d, j, d.z);
    const double xj = d.x[j], sj = d.s[j];
    const double rxs = rxs_of(d, mode, j, sigma_mu);
    double dxj, dsj;
    bool fr = false;
    if (!d.qp) {
      // solve_newton (interior_point.cpp:443-450)
      const double dj = fmax(xj, 1e-16) / fmax(sj, 1e-16);
      dxj = dj * (atdy - d.rd[j]) + rxs / fmax(sj, 1e-16);
      dsj = d.rd[j] - atdy;
    } else {
      // dx = D (r1 + A'dy); ds = (rxs - s dx)/x (qp_interior_point.cpp:2832-2844)
      fr = d.free_col[j];
      const double xf = fmax(xj, 1e-16);
      if (dxv) {  // coupled Hessian: dx = H^-1 (r1 + A'dy), solved by the caller
        dxj = dxv[j];
      } else {
        const double D = 1.0 / (d.qdiag[j] + (fr ? 0.0 : fmax(sj, 1e-16) / xf));
        const double r1 = fr ? -d.rd[j] : -d.rd[j] + rxs / xf;
        dxj = D * (r1 + atdy);
      }
      dsj = fr ? 0.0 : (rxs - sj * dxj) / xf;
    }
    dx[j] = dxj;
    ds[j] = dsj;
    if (!fr) {
      if (dxj < 0.0) rp_min = fmin(rp_min, -xj / dxj);
      if (dsj < 0.0) rd_min = fmin(rd_min, -sj / dsj);
    }
  }
  double v[2] = {rp_min, rd_min};
  const int ops[2] = {2, 2};
  if (grid_reduce<2>(v, ops, d.partials, d.counter) && threadIdx.x == 0) {
    IpmScalars* sc = d.sc;
    sc->ratio_p = v[0];
    sc->ratio_d = v[1];
    if (mode == kRhsAffine) {
      sc->alpha_p_aff = v[0];
      sc->alpha_d_aff = v[1];
    } else {
      double ap = fmin(1.0, d.tau * v[0]);
      double ad = fmin(1.0, d.tau * v[1]);
      if (d.qp && d.has_quadratic) ap = ad = fmin(ap, ad);  // common step (qp_interior_point.cpp:3095)
      sc->alpha_p = ap;
      sc->alpha_d = ad;
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_mu_aff(IpmDev d) {
  const double ap = d.sc->alpha_p_aff, ad = d.sc->alpha_d_aff;
  double acc = 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    if (d.qp && d.free_col[j]) continue;
    acc += (d.x[j] + ap * d.dxa[j]) * (d.s[j] + ad * d.dsa[j]);
  }
  double v[1] = {acc};
  const int ops[1] = {0};
  if (grid_reduce<1>(v, ops, d.partials, d.counter) && threadIdx.x == 0) {
    IpmScalars* sc = d.sc;
    const double cnt = d.qp ? d.comp_count : static_cast<double>(d.n);
    sc->mu_aff = v[0] / cnt;
    const double r = sc->mu_aff / sc->mu;
    sc->sigma = sc->mu > 0.0 ? fmin(1.0, r * r * r) : 0.0;  // (mu_aff/mu)^3 (interior_point.cpp:672-673)
  }
}

__global__ void __launch_bounds__(kThreads) k_update(IpmDev d) {
  if (d.sc->fail) {
    if (blockIdx.x == 0 && threadIdx.x == 0) d.sc->skipped = 1;
    return;
  }
  const double ap = d.sc->alpha_p, ad = d.sc->alpha_d;
  const int N = d.n > d.m ? d.n : d.m;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    if (j < d.n) {
      if (d.qp && d.free_col[j]) {
        d.x[j] += ap * d.dx[j];
      } else {
        d.x[j] = fmax(d.x[j] + ap * d.dx[j], 1e-14);
        d.s[j] = fmax(d.s[j] + ad * d.ds[j], 1e-14);
      }
    }
    if (j < d.m) d.y[j] += ad * d.dy[j];
  }
}

__global__ void __launch_bounds__(kThreads) k_start_rhs(IpmDev d) {
  for_each_row(d, [&](int p) { return d.rval[p]; }, [&](int i, double acc) { d.z[i] = d.b[i] - acc; });
}

__global__ void __launch_bounds__(kThreads) k_start_rhs_cut(IpmDev d) {
  for_each_cut_row(d, [&](int i, double acc) { d.z[i] = d.b[i] - acc; });
}

__global__ void __launch_bounds__(kThreads) k_start_point(IpmDev d) {
  const bool ok = !d.sc->fail;
  const int N = d.n > d.m ? d.n : d.m;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    if (j < d.n) {
      double x = 1.0, s = 1.0;
      if (ok) {
        const double atdy = col_dot(d, j, d.dy);
        if (!d.qp) {
          x = fmax(1.0, fabs(atdy));
          s = fmax(1.0, fabs(d.c[j] - atdy));
        } else if (d.free_col[j]) {
          x = 1.0 + atdy;
        } else {
          double qones = d.qdiag[j];  // (Q 1)_j (qp_interior_point.cpp:2933-2941)
          if (d.q_coupled) {
            qones = 0.0;
            for (int k = d.q_ptr[j]; k < d.q_ptr[j + 1]; ++k) qones += d.q_val[k];
          }
          x = fmax(1.0, fabs(atdy));
          s = fmax(1.0, fabs(qones + d.c[j] - atdy));
        }
      }
      if (d.qp && d.free_col[j]) s = 0.0;
      d.x[j] = x;
      d.s[j] = s;
    }
    if (j < d.m) d.y[j] = ok ? d.dy[j] : 0.0;
  }
}

__global__ void __launch_bounds__(kThreads) k_normal_cols(IpmDev d, const double* v, double* tmp) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    const double a = col_dot(d, j, v);
    const double xj = fmax(d.x[j], 1e-16), sj = fmax(d.s[j], 1e-16);
    double w;
    if (d.start_system) w = 1.0;
    else if (!d.qp) w = xj / sj;
    else w = 1.0 / (d.qdiag[j] + (d.free_col[j] ? 0.0 : sj / xj));
    tmp[j] = w * a;
  }
}

__global__ void __launch_bounds__(kThreads) k_normal_rows(IpmDev d, const double* v, const double* tmp, double* out,
                                                          double reg) {
  for_each_row(
      d, [&](int p) { return d.rval[p] * tmp[d.col_idx[p]]; }, [&](int i, double acc) { out[i] = acc + reg * v[i]; });
}

__global__ void __launch_bounds__(kThreads) k_normal_rows_cut(IpmDev d, const double* v, double* out, double reg) {
  for_each_cut_row(d, [&](int i, double acc) { out[i] = acc + reg * v[i]; });
}

// ---------------------------------------------------------------------------------------------
// x-space QP: K dx_x = r1_x + A_x'(Theta rp - sigma r1_w), dy = Theta (rp - A_x dx_x) - sigma r1_w,
// dw = (r1_w + sigma dy) / h_w  (the slack columns of the KKT system of solve_newton_qp,
// qp_interior_point.cpp:2832-2844, eliminated row by row)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ double h_of(const IpmDev& d, int j) {
  return fmax(d.s[j], 1e-16) / fmax(d.x[j], 1e-16);
}
__device__ __forceinline__ double r1_of(const IpmDev& d, int mode, int j, double sigma_mu) {
  const double rxs = rxs_of(d, mode, j, sigma_mu);
  if (d.free_col[j]) return -d.rd[j];
  return -d.rd[j] + rxs / fmax(d.x[j], 1e-16);
}

__global__ void __launch_bounds__(kThreads) k_xrhs_rows(IpmDev d, int mode) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < d.m; r += gridDim.x * blockDim.x) {
    const int w = d.slack_of_row[r];
    d.tr[r] = h_of(d, w) * d.rp[r] - d.sigma[r] * r1_of(d, mode, w, sigma_mu);
  }
}

__global__ void __launch_bounds__(kThreads) k_xrhs_cols(IpmDev d, int mode) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.nx; j += gridDim.x * blockDim.x) {
    const double acc = col_dot(d, j, d.tr);
    d.z[j] = (mode < 0 ? 0.0 : r1_of(d, mode, j, sigma_mu)) + acc;
  }
}

// rows: dy, dw and the slack's ds; structural columns: dx = z, ds; both ratio tests
__global__ void __launch_bounds__(kThreads) k_xdirection(IpmDev d, int mode) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  double* dx = mode == kRhsAffine ? d.dxa : d.dx;
  double* ds = mode == kRhsAffine ? d.dsa : d.ds;
  double rp_min = 1.0, rd_min = 1.0;
  const int N = d.m > d.nx ? d.m : d.nx;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < N; t += gridDim.x * blockDim.x) {
    if (t < d.m) {
      const int r = t, w = d.slack_of_row[r];
      double ax = 0.0;
      for (int p = d.row_ptr[r]; p < d.row_ptr[r + 1]; ++p) {
        const int j = d.col_idx[p];
        if (j < d.nx) ax += d.rval[p] * d.z[j];
      }
      const double hw = h_of(d, w);
      const double r1w = r1_of(d, mode, w, sigma_mu);
      const double dyr = hw * (d.rp[r] - ax) - d.sigma[r] * r1w;
      const double dw = (r1w + d.sigma[r] * dyr) / hw;
      const double xw = d.x[w], sw = d.s[w];
      const double dsw = (rxs_of(d, mode, w, sigma_mu) - sw * dw) / fmax(xw, 1e-16);
      d.dy[r] = dyr;
      dx[w] = dw;
      ds[w] = dsw;
      if (dw < 0.0) rp_min = fmin(rp_min, -xw / dw);
      if (dsw < 0.0) rd_min = fmin(rd_min, -sw / dsw);
    }
    if (t < d.nx) {
      const int j = t;
      const double dxj = d.z[j];
      const bool fr = d.free_col[j];
      const double dsj = fr ? 0.0 : (rxs_of(d, mode, j, sigma_mu) - d.s[j] * dxj) / fmax(d.x[j], 1e-16);
      dx[j] = dxj;
      ds[j] = dsj;
      if (!fr) {
        if (dxj < 0.0) rp_min = fmin(rp_min, -d.x[j] / dxj);
        if (dsj < 0.0) rd_min = fmin(rd_min, -d.s[j] / dsj);
      }
    }
  }
  double v[2] = {rp_min, rd_min};
  const int ops[2] = {2, 2};
  if (grid_reduce<2>(v, ops, d.partials, d.counter) && threadIdx.x == 0) {
    IpmScalars* sc = d.sc;
    sc->ratio_p = v[0];
    sc->ratio_d = v[1];
    if (mode == kRhsAffine) {
      sc->alpha_p_aff = v[0];
      sc->alpha_d_aff = v[1];
    } else {
      double ap = fmin(1.0, d.tau * v[0]);
      double ad = fmin(1.0, d.tau * v[1]);
      if (d.has_quadratic) ap = ad = fmin(ap, ad);  // common step (qp_interior_point.cpp:3095)
      sc->alpha_p = ap;
      sc->alpha_d = ad;
    }
  }
}

// start (qp_interior_point.cpp:2884-2891 with H = I): t = b - A 1, K = I + A_x'A_x, z = A_x' t
__global__ void __launch_bounds__(kThreads) k_xstart_rows(IpmDev d) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < d.m; r += gridDim.x * blockDim.x) {
    double acc = 0.0;
    for (int p = d.row_ptr[r]; p < d.row_ptr[r + 1]; ++p) acc += d.rval[p];
    d.tr[r] = d.b[r] - acc;
  }
}
__global__ void __launch_bounds__(kThreads) k_xstart_dy(IpmDev d) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < d.m; r += gridDim.x * blockDim.x) {
    double ax = 0.0;
    for (int p = d.row_ptr[r]; p < d.row_ptr[r + 1]; ++p) {
      const int j = d.col_idx[p];
      if (j < d.nx) ax += d.rval[p] * d.z[j];
    }
    d.dy[r] = d.tr[r] - ax;
  }
}

__global__ void __launch_bounds__(kThreads) k_xdiag(IpmDev d, int mode, double* M, int layout_ld, double* diag) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.nx; j += gridDim.x * blockDim.x) {
    const double add = mode == 0 ? 1.0 : d.qdiag[j] + (d.free_col[j] ? 0.0 : h_of(d, j));
    const int64_t pos = layout_ld > 0 ? static_cast<int64_t>(j) * layout_ld + j : j;
    M[pos] += add;
    diag[j] += add;
  }
}

// ---- coupled-Hessian QP ----
__global__ void __launch_bounds__(kThreads) k_hessian_diag(IpmDev d, int start, double* H, int ld, double* diag) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    const double xf = fmax(d.x[j], 1e-16), sf = fmax(d.s[j], 1e-16);
    const double h = d.free_col[j] ? 0.0 : (start ? 1.0 : sf / xf);
    double* hjj = H + static_cast<int64_t>(j) * ld + j;
    *hjj += h;
    diag[j] = *hjj;
  }
}

__global__ void __launch_bounds__(kThreads) k_rows_to_columns(IpmDev d, double* Y, int ld) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  for (int i = warp_row(); i < d.m; i += warps)
    for (int p = d.row_ptr[i] + lane; p < d.row_ptr[i + 1]; p += 32)
      Y[static_cast<int64_t>(i) * ld + d.col_idx[p]] = d.rval[p];
}

// one warp per lower-triangle entry (i, k), k <= i: sum over row i of A of a_ij Y[j][k]
__global__ void __launch_bounds__(kThreads) k_form_normal(IpmDev d, const double* Y, int ld_y, double* M, int ld_m,
                                                          double reg, double* diag) {
  const int lane = threadIdx.x & 31;
  const int warps = gridDim.x * (blockDim.x >> 5);
  const int64_t pairs = static_cast<int64_t>(d.m) * (d.m + 1) / 2;
  for (int64_t t = warp_row(); t < pairs; t += warps) {
    int i = static_cast<int>((sqrt(8.0 * static_cast<double>(t) + 1.0) - 1.0) * 0.5);
    while (static_cast<int64_t>(i + 1) * (i + 2) / 2 <= t) ++i;
    while (static_cast<int64_t>(i) * (i + 1) / 2 > t) --i;
    const int k = static_cast<int>(t - static_cast<int64_t>(i) * (i + 1) / 2);
    const double* yk = Y + static_cast<int64_t>(k) * ld_y;
    double acc = 0.0;
    for (int p = d.row_ptr[i] + lane; p < d.row_ptr[i + 1]; p += 32) acc += d.rval[p] * yk[d.col_idx[p]];
    acc = warp_sum(acc);
    if (lane == 0) {
      const double v = i == k ? acc + reg : acc;
      M[static_cast<int64_t>(k) * ld_m + i] = v;
      if (i == k) diag[i] = v;
    }
  }
}

__device__ __forceinline__ double hessian_r1(const IpmDev& d, int mode, int j, double sigma_mu) {
  const double rxs = rxs_of(d, mode, j, sigma_mu);
  return d.free_col[j] ? -d.rd[j] : -d.rd[j] + rxs / fmax(d.x[j], 1e-16);
}

__global__ void __launch_bounds__(kThreads) k_hessian_r1(IpmDev d, int mode, double* v) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x)
    v[j] = hessian_r1(d, mode, j, sigma_mu);
}

__global__ void __launch_bounds__(kThreads) k_rows_minus(IpmDev d, const double* v, const double* base) {
  for_each_row(
      d, [&](int p) { return d.rval[p] * v[d.col_idx[p]]; },
      [&](int i, double acc) { d.z[i] = (base ? base[i] : 0.0) - acc; });
}

__global__ void __launch_bounds__(kThreads) k_rows_minus_cut(IpmDev d, const double* base) {
  for_each_cut_row(d, [&](int i, double acc) { d.z[i] = (base ? base[i] : 0.0) - acc; });
}

__global__ void __launch_bounds__(kThreads) k_mehrotra_xt(IpmDev d, double* xt) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    const double atdy = col_dot(d, j, d.z);
    xt[j] = 1.0 + atdy;
  }
}

__global__ void __launch_bounds__(kThreads) k_mehrotra_r1(IpmDev d, const double* xt, double* r1) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    double qx = 0.0;
    if (d.q_coupled) {
      for (int k = d.q_ptr[j]; k < d.q_ptr[j + 1]; ++k) qx += d.q_val[k] * xt[d.q_idx[k]];
    } else {
      qx = d.qdiag[j] * xt[j];
    }
    r1[j] = -(d.c[j] + qx);
  }
}

__global__ void __launch_bounds__(kThreads) k_add_atz(IpmDev d, const double* r1, double* w) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    const double atz = col_dot(d, j, d.z);
    w[j] = r1[j] + atz;
  }
}

__global__ void __launch_bounds__(kThreads) k_hessian_w(IpmDev d, int mode, double* v) {
  const double sigma_mu = mode == kRhsCorrector ? d.sc->sigma * d.sc->mu : 0.0;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < d.n; j += gridDim.x * blockDim.x) {
    const double atdy = col_dot(d, j, d.z);
    v[j] = hessian_r1(d, mode, j, sigma_mu) + atdy;
  }
}

int row_blocks(int m) { return std::max(1, std::min(kMaxBlocks, ceil_div(static_cast<long long>(m) * 32, kThreads))); }
// grid of a for_each_row kernel: a warp per piece or per row, or a CTA per row
int row_blocks(const IpmDev& d) {
  if (d.row_piece) return row_blocks(d.row_pieces);
  return d.row_block ? std::max(1, std::min(kMaxBlocks, d.m)) : row_blocks(d.m);
}
int cut_blocks(const IpmDev& d) { return blocks_for(d.row_combs); }

}  // namespace

int reduction_blocks(int n) { return blocks_for(n); }

void launch_residuals(const IpmDev& d, cudaStream_t st, int* launches) {
  k_residual_rows<<<row_blocks(d), kThreads, 0, st>>>(d);
  if (d.row_combs) k_residual_rows_cut<<<1, kThreads, 0, st>>>(d);
  k_residual_cols<<<blocks_for(d.n), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += 2;
}

void launch_newton_rhs(const IpmDev& d, int mode, cudaStream_t st, int* launches) {
  if (d.coltmp) k_newton_tmp<<<blocks_for(d.n), kThreads, 0, st>>>(d, mode);
  k_newton_rhs<<<row_blocks(d), kThreads, 0, st>>>(d, mode);
  if (d.row_combs) k_newton_rhs_cut<<<cut_blocks(d), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += (d.coltmp ? 2 : 1) + (d.row_combs ? 1 : 0);
}

void launch_direction(const IpmDev& d, int mode, cudaStream_t st, int* launches) {
  k_direction<<<blocks_for(d.n), kThreads, 0, st>>>(d, mode, nullptr);
  if (mode == kRhsAffine) k_mu_aff<<<blocks_for(d.n), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += mode == kRhsAffine ? 2 : 1;
}

void launch_direction_dx(const IpmDev& d, int mode, const double* dxv, cudaStream_t st, int* launches) {
  k_direction<<<blocks_for(d.n), kThreads, 0, st>>>(d, mode, dxv);
  if (mode == kRhsAffine) k_mu_aff<<<blocks_for(d.n), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += mode == kRhsAffine ? 2 : 1;
}

void launch_update(const IpmDev& d, cudaStream_t st, int* launches) {
  k_update<<<blocks_for(std::max(d.n, d.m)), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += 1;
}

void launch_start_rhs(const IpmDev& d, cudaStream_t st, int* launches) {
  k_start_rhs<<<row_blocks(d), kThreads, 0, st>>>(d);
  if (d.row_combs) k_start_rhs_cut<<<cut_blocks(d), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += 1;
}

void launch_start_point(const IpmDev& d, cudaStream_t st, int* launches) {
  k_start_point<<<blocks_for(std::max(d.n, d.m)), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += 1;
}

void launch_newton_rhs_x(const IpmDev& d, int mode, cudaStream_t st, int* launches) {
  k_xrhs_rows<<<blocks_for(d.m), kThreads, 0, st>>>(d, mode);
  k_xrhs_cols<<<blocks_for(d.nx), kThreads, 0, st>>>(d, mode);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += 2;
}

void launch_direction_x(const IpmDev& d, int mode, cudaStream_t st, int* launches) {
  k_xdirection<<<blocks_for(std::max(d.m, d.nx)), kThreads, 0, st>>>(d, mode);
  if (mode == kRhsAffine) k_mu_aff<<<blocks_for(d.n), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += mode == kRhsAffine ? 2 : 1;
}

void launch_start_rhs_x(const IpmDev& d, cudaStream_t st, int* launches) {
  k_xstart_rows<<<blocks_for(d.m), kThreads, 0, st>>>(d);
  k_xrhs_cols<<<blocks_for(d.nx), kThreads, 0, st>>>(d, -1);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += 2;
}

void launch_start_dy_x(const IpmDev& d, cudaStream_t st, int* launches) {
  k_xstart_dy<<<blocks_for(d.m), kThreads, 0, st>>>(d);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += 1;
}

void launch_xspace_diag(const IpmDev& d, int mode, double* M, int layout_ld, double* diag, cudaStream_t st) {
  k_xdiag<<<blocks_for(d.nx), kThreads, 0, st>>>(d, mode, M, layout_ld, diag);
  SOV_LAUNCH_CHECK();
}

void launch_normal_matvec(const IpmDev& d, const double* v, double* tmp_n, double* out, double reg, cudaStream_t st) {
  k_normal_cols<<<blocks_for(d.n), kThreads, 0, st>>>(d, v, tmp_n);
  k_normal_rows<<<row_blocks(d), kThreads, 0, st>>>(d, v, tmp_n, out, reg);
  if (d.row_combs) k_normal_rows_cut<<<cut_blocks(d), kThreads, 0, st>>>(d, v, out, reg);
  SOV_LAUNCH_CHECK();
}

}  // namespace sov

namespace sov {

void launch_hessian_diag(const IpmDev& d, bool start, double* H, int ld, double* diag, cudaStream_t st) {
  k_hessian_diag<<<blocks_for(d.n), kThreads, 0, st>>>(d, start ? 1 : 0, H, ld, diag);
  SOV_LAUNCH_CHECK();
}

void launch_rows_to_columns(const IpmDev& d, double* Y, int ld, cudaStream_t st) {
  k_rows_to_columns<<<row_blocks(d.m), kThreads, 0, st>>>(d, Y, ld);
  SOV_LAUNCH_CHECK();
}

void launch_form_normal(const IpmDev& d, const double* Y, int ld_y, double* M, int ld_m, double reg, double* diag,
                        cudaStream_t st) {
  const long long pairs = static_cast<long long>(d.m) * (d.m + 1) / 2;
  k_form_normal<<<std::max(1, std::min(kMaxBlocks, ceil_div(pairs * 32, kThreads))), kThreads, 0, st>>>(
      d, Y, ld_y, M, ld_m, reg, diag);
  SOV_LAUNCH_CHECK();
}

void launch_hessian_r1(const IpmDev& d, int mode, double* v, cudaStream_t st) {
  k_hessian_r1<<<blocks_for(d.n), kThreads, 0, st>>>(d, mode, v);
  SOV_LAUNCH_CHECK();
}

void launch_rows_minus(const IpmDev& d, const double* v, const double* base, cudaStream_t st) {
  k_rows_minus<<<row_blocks(d), kThreads, 0, st>>>(d, v, base);
  if (d.row_combs) k_rows_minus_cut<<<cut_blocks(d), kThreads, 0, st>>>(d, base);
  SOV_LAUNCH_CHECK();
}

void launch_mehrotra_r1(const IpmDev& d, double* xt, double* r1, cudaStream_t st) {
  k_mehrotra_xt<<<blocks_for(d.n), kThreads, 0, st>>>(d, xt);
  k_mehrotra_r1<<<blocks_for(d.n), kThreads, 0, st>>>(d, xt, r1);
  SOV_LAUNCH_CHECK();
}

void launch_add_atz(const IpmDev& d, const double* r1, double* w, cudaStream_t st) {
  k_add_atz<<<blocks_for(d.n), kThreads, 0, st>>>(d, r1, w);
  SOV_LAUNCH_CHECK();
}

void launch_hessian_w(const IpmDev& d, int mode, double* v, cudaStream_t st) {
  k_hessian_w<<<blocks_for(d.n), kThreads, 0, st>>>(d, mode, v);
  SOV_LAUNCH_CHECK();
}

}  // namespace sov
