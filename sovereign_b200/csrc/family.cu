// family.cu -- a family of LPs sharing A, solved W at a time in lockstep (see family.cuh).
#include "family.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "engine.hpp"
#include "sparse.hpp"
#include "stdform.hpp"

namespace cg = cooperative_groups;

namespace sov {
namespace {

constexpr int kFamThreads = 256;
constexpr int kFamBlocks = 296;  // 2 CTAs per SM for the grid-stride passes (the per-LP folds read one partial per CTA)
constexpr int kWarmGiveUp = 40;  // iterations a supplied start gets before the default restart
constexpr int kNv = 3;           // reduction slots per pass
constexpr int kFamPiece = 32;    // terms per piece of the family's sparse schedule

// Per-LP scalars of one iteration (the single engine's IpmScalars for an LP).
struct FamScalars {
  double rp_max, rd_max, xs, cx, mu, p_res, d_res, gap, metric;
  double ratio_p, ratio_d, alpha_p_aff, alpha_d_aff, mu_aff, sigma, alpha_p, alpha_d;
  int fail, drops, skipped, pad;
};

struct FamDev {
  int m, n, W, G;  // rows, columns, LPs in the chunk, LPs' entries per CTA (blockDim = W * G)
  const int *row_ptr, *col_idx, *col_ptr, *row_idx;
  const double *rval, *cval;
  const double *b, *c;          // m x W, n x W (interleaved: entry-major, LP fastest)
  const double *bnorm, *cnorm;  // W
  double *x, *s, *y;
  double *dx, *ds, *dxa, *dsa, *rd, *rp, *z, *t;
  FamScalars* sc;    // W
  const int* step;   // W: 1 when the LP takes this iteration's step
  double* part;      // reduction partials: kFamBlocks x kNv x W
  double tau;
};

// The normal matrices' shared symbolic factor and schedule, values per LP (interleaved).
struct FamSparse {
  int m, levels, W;
  int tail, mt;             // dense trailing block: columns mt .. m-1, factored and solved densely
  double* Ld;               // its strict lower triangle, packed by columns (explicit zeros included)
  const int* tail_off;      // tail column q's first entry (row q + 1) in Ld
  const int *blk_src, *blk_dst;  // the block's pattern entries: index into V -> index into Ld
  int blk_n;
  const int *pivot_ptr, *pivot_col;  // the columns before the tail, per level
  double *V, *diag, *inv_d, *work, *partial;  // (m + nnz(L)) x W, m x W, m x W, m x W, slots x W
  const int *perm, *lvl_ptr, *lvl_col, *li;
  const int4 *fpiece, *fcomb, *lpiece, *lcomb, *upiece, *ucomb;
  const int *fpiece_lvl, *fcomb_lvl, *lpiece_lvl, *lcomb_lvl, *upiece_lvl, *ucomb_lvl;
  const int *up_col, *up_a, *up_b, *row_pos, *row_col;
  FamScalars* sc;
  double drop_tol;
};

struct FamAssembly {
  const int* target;  // into [D | L]
  const int* ptr;
  const int* col;
  const double* w;
  int ntargets;
};

// thread -> (first item, LP) of the grid-stride loops: items advance by gridDim.x * G
struct Lane {
  int item, k, stride;
};
__device__ __forceinline__ Lane lane_of(const FamDev& d) {
  return Lane{static_cast<int>(blockIdx.x) * d.G + static_cast<int>(threadIdx.x) / d.W,
              static_cast<int>(threadIdx.x) % d.W, static_cast<int>(gridDim.x) * d.G};
}

// Combine this thread's values over the CTA's G items per LP (in item order) and leave the CTA's
// result in part[(block * kNv + q) * W + k]. ops: 0 sum, 1 max, 2 min.
template <int NV>
__device__ void cta_partials(const FamDev& d, double (&v)[NV], const int (&ops)[NV], double* sm) {
  const int tid = threadIdx.x, bd = blockDim.x;
#pragma unroll
  for (int q = 0; q < NV; ++q) sm[q * bd + tid] = v[q];
  __syncthreads();
  if (tid < d.W) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double acc = sm[q * bd + tid];
      for (int g = 1; g < d.G; ++g) {
        const double u = sm[q * bd + g * d.W + tid];
        acc = ops[q] == 0 ? acc + u : ops[q] == 1 ? fmax(acc, u) : fmin(acc, u);
      }
      d.part[(static_cast<size_t>(blockIdx.x) * kNv + q) * d.W + tid] = acc;
    }
  }
}

// the blocks' partials of slot q for LP k, in block order
__device__ __forceinline__ double fold(const FamDev& d, int blocks, int q, int k, int op, double init) {
  double acc = init;
  for (int b = 0; b < blocks; ++b) {
    const double u = d.part[(static_cast<size_t>(b) * kNv + q) * d.W + k];
    acc = op == 0 ? acc + u : op == 1 ? fmax(acc, u) : fmin(acc, u);
  }
  return acc;
}

// ---- residuals: rp = b - A x, rd = c - (A'y + s) (interior_point.cpp:572-602) ----
__global__ void k_fam_res_rows(FamDev d) {
  extern __shared__ double sm[];
  const Lane L = lane_of(d);
  double mx = 0.0;
  for (int i = L.item; i < d.m; i += L.stride) {
    double acc = 0.0;
    for (int p = d.row_ptr[i]; p < d.row_ptr[i + 1]; ++p) acc += d.rval[p] * d.x[static_cast<size_t>(d.col_idx[p]) * d.W + L.k];
    const size_t e = static_cast<size_t>(i) * d.W + L.k;
    const double r = d.b[e] - acc;
    d.rp[e] = r;
    mx = fmax(mx, fabs(r));
  }
  double v[1] = {mx};
  const int ops[1] = {1};
  cta_partials<1>(d, v, ops, sm);
}

__global__ void k_fam_res_cols(FamDev d) {
  extern __shared__ double sm[];
  const Lane L = lane_of(d);
  double rdm = 0.0, xs = 0.0, cx = 0.0;
  for (int j = L.item; j < d.n; j += L.stride) {
    double aty = 0.0;
    for (int p = d.col_ptr[j]; p < d.col_ptr[j + 1]; ++p) aty += d.cval[p] * d.y[static_cast<size_t>(d.row_idx[p]) * d.W + L.k];
    const size_t e = static_cast<size_t>(j) * d.W + L.k;
    const double xj = d.x[e], sj = d.s[e];
    const double r = d.c[e] - (aty + sj);
    d.rd[e] = r;
    rdm = fmax(rdm, fabs(r));
    xs += xj * sj;
    cx += d.c[e] * xj;
  }
  double v[3] = {rdm, xs, cx};
  const int ops[3] = {1, 0, 0};
  cta_partials<3>(d, v, ops, sm);
}

// one thread per LP: rows' and columns' partials (two part buffers) into the scalars
__global__ void k_fam_res_final(FamDev d, const double* rows_part, int rows_blocks, int cols_blocks) {
  const int k = threadIdx.x;
  if (k >= d.W) return;
  double rpm = 0.0;
  for (int b = 0; b < rows_blocks; ++b) rpm = fmax(rpm, rows_part[(static_cast<size_t>(b) * kNv) * d.W + k]);
  const double rdm = fold(d, cols_blocks, 0, k, 1, 0.0);
  const double xs = fold(d, cols_blocks, 1, k, 0, 0.0);
  const double cx = fold(d, cols_blocks, 2, k, 0, 0.0);
  FamScalars& sc = d.sc[k];
  sc.rp_max = rpm;
  sc.rd_max = rdm;
  sc.xs = xs;
  sc.cx = cx;
  sc.p_res = rpm / d.bnorm[k];
  sc.mu = xs / static_cast<double>(d.n);
  sc.d_res = rdm / d.cnorm[k];
  sc.gap = fabs(xs) / (1.0 + fabs(cx));
  sc.metric = fmax(sc.p_res, fmax(sc.d_res, sc.gap));
}

// ---- Newton step (interior_point.cpp:418-452, 640-690) ----
// rxs of the current mode: affine -x s; corrector -x s - dxa dsa + sigma mu
__device__ __forceinline__ double fam_rxs(const FamDev& d, int mode, size_t e, double sigma_mu) {
  const double xj = d.x[e], sj = d.s[e];
  if (mode == 0) return -xj * sj;
  return -xj * sj - d.dxa[e] * d.dsa[e] + sigma_mu;
}

// t = d rd - rxs / s per column (d = x/s with the 1e-16 floors)
__global__ void k_fam_newton_tmp(FamDev d, int mode) {
  const Lane L = lane_of(d);
  const double sigma_mu = mode == 1 ? d.sc[L.k].sigma * d.sc[L.k].mu : 0.0;
  for (int j = L.item; j < d.n; j += L.stride) {
    const size_t e = static_cast<size_t>(j) * d.W + L.k;
    const double xj = fmax(d.x[e], 1e-16), sj = fmax(d.s[e], 1e-16);
    d.t[e] = (xj / sj) * d.rd[e] - fam_rxs(d, mode, e, sigma_mu) / sj;
  }
}

// z = rp + A t
__global__ void k_fam_newton_rhs(FamDev d) {
  const Lane L = lane_of(d);
  for (int i = L.item; i < d.m; i += L.stride) {
    double acc = 0.0;
    for (int p = d.row_ptr[i]; p < d.row_ptr[i + 1]; ++p) acc += d.rval[p] * d.t[static_cast<size_t>(d.col_idx[p]) * d.W + L.k];
    const size_t e = static_cast<size_t>(i) * d.W + L.k;
    d.z[e] = d.rp[e] + acc;
  }
}

// dx = d (A'dy - rd) + rxs / s, ds = rd - A'dy with dy = z; ratio tests (step_to_bound from 1)
__global__ void k_fam_direction(FamDev d, int mode) {
  extern __shared__ double sm[];
  const Lane L = lane_of(d);
  const double sigma_mu = mode == 1 ? d.sc[L.k].sigma * d.sc[L.k].mu : 0.0;
  double* dxo = mode == 0 ? d.dxa : d.dx;
  double* dso = mode == 0 ? d.dsa : d.ds;
  double rp_min = 1.0, rd_min = 1.0;
  for (int j = L.item; j < d.n; j += L.stride) {
    double atdy = 0.0;
    for (int p = d.col_ptr[j]; p < d.col_ptr[j + 1]; ++p) atdy += d.cval[p] * d.z[static_cast<size_t>(d.row_idx[p]) * d.W + L.k];
    const size_t e = static_cast<size_t>(j) * d.W + L.k;
    const double xj = d.x[e], sj = d.s[e];
    const double rxs = fam_rxs(d, mode, e, sigma_mu);
    const double dj = fmax(xj, 1e-16) / fmax(sj, 1e-16);
    const double dxj = dj * (atdy - d.rd[e]) + rxs / fmax(sj, 1e-16);
    const double dsj = d.rd[e] - atdy;
    dxo[e] = dxj;
    dso[e] = dsj;
    if (dxj < 0.0) rp_min = fmin(rp_min, -xj / dxj);
    if (dsj < 0.0) rd_min = fmin(rd_min, -sj / dsj);
  }
  double v[2] = {rp_min, rd_min};
  const int ops[2] = {2, 2};
  cta_partials<2>(d, v, ops, sm);
}

__global__ void k_fam_direction_final(FamDev d, int mode, int blocks) {
  const int k = threadIdx.x;
  if (k >= d.W) return;
  const double rp = fold(d, blocks, 0, k, 2, 1.0), rdd = fold(d, blocks, 1, k, 2, 1.0);
  FamScalars& sc = d.sc[k];
  sc.ratio_p = rp;
  sc.ratio_d = rdd;
  if (mode == 0) {
    sc.alpha_p_aff = rp;
    sc.alpha_d_aff = rdd;
  } else {
    sc.alpha_p = fmin(1.0, d.tau * rp);
    sc.alpha_d = fmin(1.0, d.tau * rdd);
  }
}

// mu_aff = sum (x + ap dxa)(s + ad dsa) / n, sigma = (mu_aff / mu)^3 (interior_point.cpp:660-673)
__global__ void k_fam_mu_aff(FamDev d) {
  extern __shared__ double sm[];
  const Lane L = lane_of(d);
  const double ap = d.sc[L.k].alpha_p_aff, ad = d.sc[L.k].alpha_d_aff;
  double acc = 0.0;
  for (int j = L.item; j < d.n; j += L.stride) {
    const size_t e = static_cast<size_t>(j) * d.W + L.k;
    acc += (d.x[e] + ap * d.dxa[e]) * (d.s[e] + ad * d.dsa[e]);
  }
  double v[1] = {acc};
  const int ops[1] = {0};
  cta_partials<1>(d, v, ops, sm);
}

__global__ void k_fam_mu_final(FamDev d, int blocks) {
  const int k = threadIdx.x;
  if (k >= d.W) return;
  FamScalars& sc = d.sc[k];
  sc.mu_aff = fold(d, blocks, 0, k, 0, 0.0) / static_cast<double>(d.n);
  const double r = sc.mu_aff / sc.mu;
  sc.sigma = sc.mu > 0.0 ? fmin(1.0, r * r * r) : 0.0;
}

// x, s, y step (interior_point.cpp:692-699); an LP whose factorization failed is not moved
__global__ void k_fam_update(FamDev d) {
  const Lane L = lane_of(d);
  const int k = L.k;
  if (!d.step[k]) return;
  const FamScalars& sc = d.sc[k];
  if (sc.fail) {
    if (L.item == 0) d.sc[k].skipped = 1;
    return;
  }
  const double ap = sc.alpha_p, ad = sc.alpha_d;
  const int N = d.n > d.m ? d.n : d.m;
  for (int j = L.item; j < N; j += L.stride) {
    const size_t e = static_cast<size_t>(j) * d.W + k;
    if (j < d.n) {
      d.x[e] = fmax(d.x[e] + ap * d.dx[e], 1e-14);
      d.s[e] = fmax(d.s[e] + ad * d.ds[e], 1e-14);
    }
    if (j < d.m) d.y[e] += ad * d.z[e];
  }
}

// ---- Mehrotra-like start (interior_point.cpp:488-506): A A' dy = b - A 1 ----
__global__ void k_fam_start_rhs(FamDev d) {
  const Lane L = lane_of(d);
  for (int i = L.item; i < d.m; i += L.stride) {
    double acc = 0.0;
    for (int p = d.row_ptr[i]; p < d.row_ptr[i + 1]; ++p) acc += d.rval[p];
    const size_t e = static_cast<size_t>(i) * d.W + L.k;
    d.z[e] = d.b[e] - acc;
  }
}

// x = max(1, |A'dy|), s = max(1, |c - A'dy|), y = dy (all 1 / 0 when the factorization failed),
// into (x, y, s) = the pointers given (the start is kept for restarts)
__global__ void k_fam_start_point(FamDev d, double* x, double* y, double* s) {
  const Lane L = lane_of(d);
  const bool ok = !d.sc[L.k].fail;
  const int N = d.n > d.m ? d.n : d.m;
  for (int j = L.item; j < N; j += L.stride) {
    const size_t e = static_cast<size_t>(j) * d.W + L.k;
    if (j < d.n) {
      double xs = 1.0, ss = 1.0;
      if (ok) {
        double atdy = 0.0;
        for (int p = d.col_ptr[j]; p < d.col_ptr[j + 1]; ++p) atdy += d.cval[p] * d.z[static_cast<size_t>(d.row_idx[p]) * d.W + L.k];
        xs = fmax(1.0, fabs(atdy));
        ss = fmax(1.0, fabs(d.c[e] - atdy));
      }
      x[e] = xs;
      s[e] = ss;
    }
    if (j < d.m) y[e] = ok ? d.z[e] : 0.0;
  }
}

// dst = src for the LPs with mask[k] (count entries per LP)
__global__ void k_fam_copy(int count, int W, const int* mask, double* dst, const double* src) {
  const long long total = static_cast<long long>(count) * W;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x)
    if (mask[t % W]) dst[t] = src[t];
}

// ---- moving one LP's vector between its slot of the interleaved arrays and contiguous storage ----
// slot column slot[i] of dst <- src + i * len, for i < count
__global__ void k_slot_put(double* dst, int len, int W, const int* slot, const double* src, int count) {
  const long long total = static_cast<long long>(count) * len;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / len), e = static_cast<int>(t % len);
    dst[static_cast<size_t>(e) * W + slot[i]] = src[t];
  }
}

// dst + i * len <- slot column slot[i] of src, for i < count
__global__ void k_slot_get(double* dst, int len, int W, const int* slot, const double* src, int count) {
  const long long total = static_cast<long long>(count) * len;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(t / len), e = static_cast<int>(t % len);
    dst[t] = src[static_cast<size_t>(e) * W + slot[i]];
  }
}

__global__ void k_fill(double* v, long long count, double value) {
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < count;
       t += static_cast<long long>(gridDim.x) * blockDim.x)
    v[t] = value;
}

// ---- normal matrices A D_k A' + 1e-12 I into the shared pattern (LP weights x/s, or 1) ----
__global__ void k_fam_assemble(FamAssembly am, FamDev d, FamSparse f, int ones) {
  const long long total = static_cast<long long>(am.ntargets) * d.W;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int q = static_cast<int>(t / d.W), k = static_cast<int>(t % d.W);
    double acc = 0.0;
    for (int p = am.ptr[q]; p < am.ptr[q + 1]; ++p) {
      const size_t e = static_cast<size_t>(am.col[p]) * d.W + k;
      acc += am.w[p] * (ones ? 1.0 : fmax(d.x[e], 1e-16) / fmax(d.s[e], 1e-16));
    }
    const int tg = am.target[q];
    if (tg < f.m) {
      acc += 1e-12;  // kNormalEqRegularization (interior_point.cpp:103)
      f.diag[static_cast<size_t>(tg) * d.W + k] = acc;
    }
    f.V[static_cast<size_t>(tg) * d.W + k] = acc;
  }
}

// ---- L D L' of every LP's normal matrix on the shared schedule (sparse_gpu.cu's walk, one
// thread per (work piece, LP); each piece's terms summed in order) ----
__global__ void __launch_bounds__(kFamThreads) k_fam_factor(FamSparse f) {
  cg::grid_group g = cg::this_grid();
  const long long rank = g.thread_rank(), size = g.size();
  const int W = f.W;
  for (int h = 0; h < f.levels; ++h) {
    const long long cols = static_cast<long long>(f.pivot_ptr[h + 1] - f.pivot_ptr[h]) * W;
    for (long long t = rank; t < cols; t += size) {
      const int k = static_cast<int>(t % W);
      const int c = f.pivot_col[f.pivot_ptr[h] + static_cast<int>(t / W)];
      const size_t e = static_cast<size_t>(c) * W + k;
      const double p = f.V[e];
      const bool finite = fabs(p) <= 1.7976931348623157e308;
      // dependent row: pivot <= 1e-13 |assembled diagonal| (sparse_ldlt.cpp:165-173)
      const bool drop = !(finite && p > f.drop_tol * fabs(f.diag[e]));
      if (drop) atomicAdd(&f.sc[k].drops, 1);
      if (!finite) atomicExch(&f.sc[k].fail, 1);
      f.inv_d[e] = 1.0 / (drop ? 1e128 : p);
    }
    g.sync();
    const long long pieces = static_cast<long long>(f.fpiece_lvl[h + 1] - f.fpiece_lvl[h]) * W;
    for (long long t = rank; t < pieces; t += size) {
      const int k = static_cast<int>(t % W);
      const int4 pc = f.fpiece[f.fpiece_lvl[h] + static_cast<int>(t / W)];
      double acc = 0.0;
      for (int u = pc.x; u < pc.y; ++u)
        acc += f.V[static_cast<size_t>(f.m + f.up_a[u]) * W + k] * f.V[static_cast<size_t>(f.m + f.up_b[u]) * W + k] *
               f.inv_d[static_cast<size_t>(f.up_col[u]) * W + k];
      if (pc.w < 0) f.V[static_cast<size_t>(pc.z) * W + k] -= acc;
      else f.partial[static_cast<size_t>(pc.w) * W + k] = acc;
    }
    if (f.fcomb_lvl[h + 1] > f.fcomb_lvl[h]) {  // uniform over the grid
      g.sync();
      const long long combs = static_cast<long long>(f.fcomb_lvl[h + 1] - f.fcomb_lvl[h]) * W;
      for (long long t = rank; t < combs; t += size) {
        const int k = static_cast<int>(t % W);
        const int4 cb = f.fcomb[f.fcomb_lvl[h] + static_cast<int>(t / W)];
        double acc = 0.0;
        for (int q = 0; q < cb.z; ++q) acc += f.partial[static_cast<size_t>(cb.y + q) * W + k];
        f.V[static_cast<size_t>(cb.x) * W + k] -= acc;
      }
    }
    g.sync();
  }
}

// ---- the dense tail (the root clique of the elimination tree), factored per LP by panels of
// kPanel columns: the panel's diagonal block, the rows below it, then the trailing block's
// update -- the same operations per entry, in the same column order, as the level schedule ----
constexpr int kPanel = 16;       // columns per panel of the dense factorization
constexpr int kSolvePanel = 32;  // rows per panel of the dense solves: a warp's lanes

// the block's values after the level schedule, scattered from the pattern into the dense storage
__global__ void k_tail_scatter(FamSparse f) {
  const long long total = static_cast<long long>(f.blk_n) * f.W;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int q = static_cast<int>(t / f.W), lp = static_cast<int>(t % f.W);
    f.Ld[static_cast<size_t>(f.blk_dst[q]) * f.W + lp] = f.V[static_cast<size_t>(f.blk_src[q]) * f.W + lp];
  }
}

__device__ __forceinline__ size_t tail_at(const FamSparse& f, int a, int q, int lp) {  // L~_aq, a > q, in Ld
  return static_cast<size_t>(f.tail_off[q] + (a - q - 1)) * f.W + lp;
}

// one CTA of P x W threads (row r of the panel, LP): each thread holds its row of the panel's
// diagonal block in registers; step j's column is exchanged through shared memory
__global__ void k_tail_diag(FamSparse f, int j0, int j1) {
  __shared__ double colv[kPanel][kFamilyWidth];
  __shared__ double invs[kFamilyWidth];
  const int W = f.W, P = j1 - j0;
  const int r = static_cast<int>(threadIdx.x) / W, lp = static_cast<int>(threadIdx.x) % W;
  const bool on = r < P;
  double a[kPanel];  // a[c] = L~_rc (c < r), a[r] = D_r
#pragma unroll
  for (int c = 0; c < kPanel; ++c)
    a[c] = (on && c <= r) ? (c == r ? f.V[static_cast<size_t>(f.mt + j0 + r) * W + lp] : f.Ld[tail_at(f, j0 + r, j0 + c, lp)])
                          : 0.0;
#pragma unroll
  for (int j = 0; j < kPanel; ++j) {
    if (j < P) {  // uniform over the CTA
      if (on && r == j) {
        const size_t e = static_cast<size_t>(f.mt + j0 + j) * W + lp;
        const double p = a[j];
        const bool finite = fabs(p) <= 1.7976931348623157e308;
        const bool drop = !(finite && p > f.drop_tol * fabs(f.diag[e]));
        if (drop) atomicAdd(&f.sc[lp].drops, 1);
        if (!finite) atomicExch(&f.sc[lp].fail, 1);
        const double inv = 1.0 / (drop ? 1e128 : p);
        f.inv_d[e] = inv;
        invs[lp] = inv;
      }
      if (on && r > j) colv[r][lp] = a[j];
      __syncthreads();
      if (on && r > j) {
        const double lrj = a[j], inv = invs[lp];
#pragma unroll
        for (int c = 0; c < kPanel; ++c)
          if (c > j && c <= r) a[c] -= lrj * colv[c][lp] * inv;
      }
      __syncthreads();
    }
  }
  if (on) {
#pragma unroll
    for (int c = 0; c < kPanel; ++c) {
      if (c < r) f.Ld[tail_at(f, j0 + r, j0 + c, lp)] = a[c];
      if (c == r) f.V[static_cast<size_t>(f.mt + j0 + r) * W + lp] = a[c];
    }
  }
}

// rows a >= j1 of the panel's columns: the in-panel recurrence on the row held in registers
__global__ void k_tail_rows(FamSparse f, int j0, int j1) {
  const int W = f.W, P = j1 - j0;
  const long long total = static_cast<long long>(f.tail - j1) * W;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int a = j1 + static_cast<int>(t / W), lp = static_cast<int>(t % W);
    double l[kPanel];
#pragma unroll
    for (int c = 0; c < kPanel; ++c) l[c] = c < P ? f.Ld[tail_at(f, a, j0 + c, lp)] : 0.0;
#pragma unroll
    for (int j = 1; j < kPanel; ++j) {
      if (j >= P) break;
      double v = l[j];
#pragma unroll
      for (int c = 0; c < kPanel; ++c) {
        if (c >= j) break;
        v -= l[c] * f.Ld[tail_at(f, j0 + j, j0 + c, lp)] * f.inv_d[static_cast<size_t>(f.mt + j0 + c) * W + lp];
      }
      l[j] = v;
    }
#pragma unroll
    for (int c = 0; c < kPanel; ++c)
      if (c < P) f.Ld[tail_at(f, a, j0 + c, lp)] = l[c];
  }
}

// the trailing block: entry (a, b), j1 <= b <= a, takes the panel's rank-P update; a thread per
// 4 x 4 tile of entries and LP (8 loads of L~ per column of the panel for 16 products)
__global__ void k_tail_update(FamSparse f, int j0, int j1) {
  const int W = f.W, P = j1 - j0, n = f.tail - j1;
  const long long nt = (n + 3) / 4, tiles = nt * (nt + 1) / 2, total = tiles * W;
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < total;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long tp = t / W;
    const int lp = static_cast<int>(t % W);
    long long ti = static_cast<long long>((sqrt(8.0 * static_cast<double>(tp) + 1.0) - 1.0) * 0.5);
    while (ti * (ti + 1) / 2 > tp) --ti;
    while ((ti + 1) * (ti + 2) / 2 <= tp) ++ti;
    const int a0 = j1 + 4 * static_cast<int>(ti), b0 = j1 + 4 * static_cast<int>(tp - ti * (ti + 1) / 2);
    double acc[4][4];
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[q][r] = 0.0;
    for (int c = 0; c < P; ++c) {
      const int col = j0 + c;
      const double inv = f.inv_d[static_cast<size_t>(f.mt + col) * W + lp];
      double la[4], lb[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        la[q] = a0 + q < f.tail ? f.Ld[tail_at(f, a0 + q, col, lp)] * inv : 0.0;
        lb[q] = b0 + q < f.tail ? f.Ld[tail_at(f, b0 + q, col, lp)] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[q][r] += la[q] * lb[r];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int a = a0 + q, b = b0 + r;
        if (a >= f.tail || b > a) continue;
        if (a == b) f.V[static_cast<size_t>(f.mt + a) * W + lp] -= acc[q][r];
        else f.Ld[tail_at(f, a, b, lp)] -= acc[q][r];
      }
  }
}

// L D L' w = z for every LP, z (original row order, interleaved) in place
__global__ void __launch_bounds__(kFamThreads) k_fam_solve(FamSparse f, double* z) {
  cg::grid_group g = cg::this_grid();
  const long long rank = g.thread_rank(), size = g.size();
  const int W = f.W;
  const long long mw = static_cast<long long>(f.m) * W;
  for (long long t = rank; t < mw; t += size)
    f.work[t] = z[static_cast<size_t>(f.perm[t / W]) * W + t % W];
  g.sync();
  const int fwd_levels = f.levels + (f.tail > 0 ? 1 : 0);  // + the tail rows' sums before the tail
  for (int h = 0; h < fwd_levels; ++h) {
    const long long pieces = static_cast<long long>(f.lpiece_lvl[h + 1] - f.lpiece_lvl[h]) * W;
    for (long long t = rank; t < pieces; t += size) {
      const int k = static_cast<int>(t % W);
      const int4 pc = f.lpiece[f.lpiece_lvl[h] + static_cast<int>(t / W)];
      double acc = 0.0;
      for (int q = pc.x; q < pc.y; ++q) {
        const size_t c = static_cast<size_t>(f.row_col[q]) * W + k;
        acc += f.V[static_cast<size_t>(f.m + f.row_pos[q]) * W + k] * f.inv_d[c] * f.work[c];
      }
      if (pc.w < 0) f.work[static_cast<size_t>(pc.z) * W + k] -= acc;
      else f.partial[static_cast<size_t>(pc.w) * W + k] = acc;
    }
    if (f.lcomb_lvl[h + 1] > f.lcomb_lvl[h]) {
      g.sync();
      const long long combs = static_cast<long long>(f.lcomb_lvl[h + 1] - f.lcomb_lvl[h]) * W;
      for (long long t = rank; t < combs; t += size) {
        const int k = static_cast<int>(t % W);
        const int4 cb = f.lcomb[f.lcomb_lvl[h] + static_cast<int>(t / W)];
        double acc = 0.0;
        for (int q = 0; q < cb.z; ++q) acc += f.partial[static_cast<size_t>(cb.y + q) * W + k];
        f.work[static_cast<size_t>(cb.x) * W + k] -= acc;
      }
    }
    g.sync();
  }
  if (f.tail > 0) {
    // The dense tail by panels of kSolvePanel (32) rows. Forward: the panel's triangle, a warp per LP with
    // lane r holding row j0 + r (y_j / D_j broadcast by shuffle), then every row below the panel
    // takes the panel's terms (a thread per row and LP). Backward, panels in reverse: the
    // triangle the same way from its last row, then every row above takes the panel's x terms.
    // Every barrier is reached by the whole grid.
    const int T = f.tail, mt = f.mt, lane = threadIdx.x & 31;
    const long long gwarp = rank >> 5, gwarps = size >> 5;
    auto w_at = [&](int a, int lp) { return static_cast<size_t>(mt + a) * W + lp; };
    for (int j0 = 0; j0 < T; j0 += kSolvePanel) {
      const int P = min(T, j0 + kSolvePanel) - j0, j1 = j0 + P;
      for (long long wl = gwarp; wl < W; wl += gwarps) {
        const int lp = static_cast<int>(wl);
        const bool on = lane < P;
        double y = on ? f.work[w_at(j0 + lane, lp)] : 0.0;
        const double inv = on ? f.inv_d[w_at(j0 + lane, lp)] : 0.0;
        for (int j = 0; j < P; ++j) {
          const double coef = __shfl_sync(0xffffffffu, y * inv, j);
          if (on && lane > j) y -= f.Ld[tail_at(f, j0 + lane, j0 + j, lp)] * coef;
        }
        if (on) f.work[w_at(j0 + lane, lp)] = y;
      }
      g.sync();
      for (long long t = rank; t < static_cast<long long>(T - j1) * W; t += size) {
        const int a = j1 + static_cast<int>(t / W), lp = static_cast<int>(t % W);
        double acc = 0.0;
        for (int j = j0; j < j1; ++j) acc += f.Ld[tail_at(f, a, j, lp)] * f.work[w_at(j, lp)] * f.inv_d[w_at(j, lp)];
        f.work[w_at(a, lp)] -= acc;
      }
      g.sync();
    }
    const int last = (T - 1) / kSolvePanel * kSolvePanel;
    for (int j0 = last; j0 >= 0; j0 -= kSolvePanel) {
      const int P = min(T, j0 + kSolvePanel) - j0;
      for (long long wl = gwarp; wl < W; wl += gwarps) {
        const int lp = static_cast<int>(wl);
        const bool on = lane < P;
        double y = on ? f.work[w_at(j0 + lane, lp)] : 0.0;
        const double inv = on ? f.inv_d[w_at(j0 + lane, lp)] : 0.0;
        for (int i = P - 1; i >= 0; --i) {
          const double xi = __shfl_sync(0xffffffffu, y * inv, i);
          if (lane == i) y = xi;
          if (on && lane < i) y -= f.Ld[tail_at(f, j0 + i, j0 + lane, lp)] * xi;
        }
        if (on) f.work[w_at(j0 + lane, lp)] = y;
      }
      g.sync();
      for (long long t = rank; t < static_cast<long long>(j0) * W; t += size) {
        const int k = static_cast<int>(t / W), lp = static_cast<int>(t % W);
        double acc = 0.0;
        for (int i = j0; i < j0 + P; ++i) acc += f.Ld[tail_at(f, i, k, lp)] * f.work[w_at(i, lp)];
        f.work[w_at(k, lp)] -= acc;
      }
      g.sync();
    }
  }
  for (int h = f.levels - 1; h >= 0; --h) {
    const long long pieces = static_cast<long long>(f.upiece_lvl[h + 1] - f.upiece_lvl[h]) * W;
    for (long long t = rank; t < pieces; t += size) {
      const int k = static_cast<int>(t % W);
      const int4 pc = f.upiece[f.upiece_lvl[h] + static_cast<int>(t / W)];
      double acc = 0.0;
      for (int p = pc.x; p < pc.y; ++p)
        acc += f.V[static_cast<size_t>(f.m + p) * W + k] * f.work[static_cast<size_t>(f.li[p]) * W + k];
      const size_t e = static_cast<size_t>(pc.z) * W + k;
      if (pc.w < 0) f.work[e] = (f.work[e] - acc) * f.inv_d[e];
      else f.partial[static_cast<size_t>(pc.w) * W + k] = acc;
    }
    if (f.ucomb_lvl[h + 1] > f.ucomb_lvl[h]) {
      g.sync();
      const long long combs = static_cast<long long>(f.ucomb_lvl[h + 1] - f.ucomb_lvl[h]) * W;
      for (long long t = rank; t < combs; t += size) {
        const int k = static_cast<int>(t % W);
        const int4 cb = f.ucomb[f.ucomb_lvl[h] + static_cast<int>(t / W)];
        double acc = 0.0;
        for (int q = 0; q < cb.z; ++q) acc += f.partial[static_cast<size_t>(cb.y + q) * W + k];
        const size_t e = static_cast<size_t>(cb.x) * W + k;
        f.work[e] = (f.work[e] - acc) * f.inv_d[e];
      }
    }
    g.sync();
  }
  for (long long t = rank; t < mw; t += size) z[static_cast<size_t>(f.perm[t / W]) * W + t % W] = f.work[t];
}

// ---------------------------------------------------------------------------------------------
// host side

template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    free_();
    n = count;
    SOV_CUDA(cudaMalloc(&p, sizeof(T) * std::max<size_t>(1, count)));
  }
  void put(const std::vector<T>& h, cudaStream_t st) {
    alloc(h.size());
    if (!h.empty()) SOV_CUDA(cudaMemcpyAsync(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st));
  }
  void free_() {
    if (p) cudaFree(p);
    p = nullptr;
  }
  ~Buf() { free_(); }
};

// the arrays a family shares, compared entry by entry (null bounds are the defaults)
bool same_structure(const sov_model& a, const sov_model& b) {
  if (a.n != b.n || a.m != b.m || a.maximize != b.maximize) return false;
  if (!std::equal(a.col_ptr, a.col_ptr + a.n + 1, b.col_ptr)) return false;
  const int nnz = a.col_ptr[a.n];
  if (!std::equal(a.row_idx, a.row_idx + nnz, b.row_idx) || !std::equal(a.values, a.values + nnz, b.values))
    return false;
  if (!std::equal(a.sense, a.sense + a.m, b.sense)) return false;
  auto bounds = [&](const double* x, const double* y, double def) {
    for (int j = 0; j < a.n; ++j)
      if ((x ? x[j] : def) != (y ? y[j] : def)) return false;
    return true;
  };
  return bounds(a.lb, b.lb, 0.0) && bounds(a.ub, b.ub, 1e30);
}

// what the chunk loop keeps per LP (the single engine's per-solve state, Engine::run)
struct LpState {
  int idx = -1;
  sov_options o{};
  bool active = true, warm_used = false, captured = false, optimal = false;
  int best_it = 0, stale = 0, factorizations = 0, its = 0;
  double best_metric = INFINITY, best_gap = INFINITY, best_p = INFINITY, best_d = INFINITY;
  double gap = 0, p_res = 0, d_res = 0;
  std::string msg;
  sov_diagnostics dg{};
};

class Family {
 public:
  Family(int count, const sov_model* models, const sov_options* opt, int opt_stride, sov_result* results)
      : count_(count), models_(models), results_(results) {
    opts_.resize(count);
    for (int k = 0; k < count; ++k) {
      if (!opt) sov_default_lp_options(&opts_[k]);
      else opts_[k] = *reinterpret_cast<const sov_options*>(reinterpret_cast<const char*>(opt) +
                                                          static_cast<size_t>(opt_stride) * k);
    }
  }
  ~Family() {
    if (st_) cudaStreamDestroy(st_);
    if (hsc_) cudaFreeHost(hsc_);
  }
  int run();

 private:
  void setup_shared(const StdForm& f);
  void solve_wave(const std::vector<int>& lps);
  // one LP's result from its vectors (contiguous; cx/cy/cs null unless captured)
  void publish(LpState& l, const double* x, const double* y, const double* s, const double* cx, const double* cy,
               const double* cs, double seconds);
  void put_slots(double* dst, int len, const int* slots, const double* src, int count);
  void get_slots(double* dst, int len, const int* slots, const double* src, int count);
  std::string describe() const;
  // launches over (entries, LPs)
  int grid_for(int items) const { return std::max(1, std::min(kFamBlocks, (items + dev_.G - 1) / dev_.G)); }
  void residuals();
  void factor();
  void solve(double* z);
  void assemble(bool ones);
  void copy(int entries, const int* mask_dev, double* dst, const double* src);

  int count_;
  const sov_model* models_;
  sov_result* results_;
  std::vector<sov_options> opts_;
  std::vector<StdForm> forms_;
  cudaStream_t st_ = nullptr;
  int sms_ = 148, per_sm_factor_ = 1, per_sm_solve_ = 1;
  // shared structure
  SparseSymbolic sym_;
  Buf<int> row_ptr_, col_idx_, col_ptr_, row_idx_, asm_target_, asm_ptr_, asm_col_;
  Buf<double> rval_, cval_, asm_w_;
  Buf<int> perm_, lvl_ptr_, lvl_col_, li_, up_col_, up_a_, up_b_, row_pos_, row_col_;
  Buf<int> fpl_, fcl_, lpl_, lcl_, upl_, ucl_, tail_off_, pivot_ptr_, pivot_col_, blk_src_, blk_dst_;
  Buf<double> Ld_;
  int tail_ = 0, blk_n_ = 0;
  size_t ld_size_ = 0;
  static constexpr int kMinTail = 32;              // smaller blocks stay in the level schedule
  static constexpr size_t kWave = 2048;            // LPs whose data and start points sit on the device
  static constexpr double kSparseTermCost = 10.0;  // a scheduled rank-1 term, in dense multiply-adds
  Buf<int4> fp_, fc_, lpc_, lc_, upc_, uc_;
  // per chunk (capacity kFamilyWidth LPs)
  Buf<double> b_, c_, bnorm_, cnorm_, x_, s_, y_, dx_, ds_, dxa_, dsa_, rd_, rp_, z_, t_;
  Buf<double> x0_, y0_, s0_, bx_, by_, bs_, cx_, cy_, cs_, part_, part_rows_;
  Buf<double> V_, diag_, inv_d_, work_, partial_;
  Buf<FamScalars> sc_;
  Buf<int> step_, mask_;
  FamScalars* hsc_ = nullptr;
  FamDev dev_{};
  FamSparse sp_{};
  FamAssembly am_{};
  int slots_ = 1;
};

int Family::run() {
  for (int k = 1; k < count_; ++k)
    if (!same_structure(models_[0], models_[k]))
      throw std::invalid_argument("sov_lp_solve_family: LP " + std::to_string(k) +
                                  " does not share the first LP's constraint matrix, bounds and row senses");
  for (int k = 1; k < count_; ++k)
    if (opts_[k].enable_scaling != opts_[0].enable_scaling ||
        opts_[k].fraction_to_boundary != opts_[0].fraction_to_boundary)
      throw std::invalid_argument("sov_lp_solve_family: every LP of a family takes the same scaling option and "
                                  "fraction to the boundary");
  SOV_CUDA(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
  // standard forms on the host (several threads); their shared part is checked against the first
  forms_.resize(count_);
  std::vector<std::string> errors(count_);
  {
    const int threads = std::max(1, std::min<int>(16, std::thread::hardware_concurrency()));
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
      pool.emplace_back([&, t] {
        for (int k = t; k < count_; k += threads) {
          try {
            forms_[k] = build_std_form(models_[k], false, opts_[k].enable_scaling != 0);
          } catch (const std::exception& e) {
            errors[k] = e.what();
          }
        }
      });
    for (auto& th : pool) th.join();
  }
  std::vector<int> members, singles;
  int first = -1;
  for (int k = 0; k < count_; ++k) {
    const StdForm& f = forms_[k];
    if (!errors[k].empty() || f.m <= 0 || f.n <= 0) {
      singles.push_back(k);
      continue;
    }
    if (first < 0) first = k;
    const StdForm& f0 = forms_[first];
    const bool shared = f.n == f0.n && f.m == f0.m && f.col_ptr == f0.col_ptr && f.row_idx == f0.row_idx &&
                        f.val == f0.val && f.col_scale == f0.col_scale && f.row_scale == f0.row_scale;
    (shared ? members : singles).push_back(k);
  }
  // LPs the family path does not take (no rows, a failed standard form, a scaling of their own):
  // the single engine, one by one
  for (int k : singles) {
    sov_result* r = &results_[k];
    if (!errors[k].empty()) {
      r->status = SOV_ERROR;
      r->has_objective_value = 0;
      std::snprintf(r->message, sizeof(r->message), "IPM error: %s", errors[k].c_str());
      continue;
    }
    const int rc = sov_lp_solve(&models_[k], &opts_[k], r);
    if (rc != SOV_OK && rc != SOV_E_ARGUMENT) return rc;
  }
  if (members.empty()) return SOV_OK;
  setup_shared(forms_[members[0]]);
  // waves of at most kWave LPs (their data and start points sit on the device); inside a wave
  // the W slots are refilled as LPs finish
  for (size_t c0 = 0; c0 < members.size(); c0 += kWave) {
    const size_t c1 = std::min(members.size(), c0 + kWave);
    solve_wave(std::vector<int>(members.begin() + c0, members.begin() + c1));
  }
  return SOV_OK;
}

void Family::setup_shared(const StdForm& f) {
  // the normal matrices' pattern, its order and symbolic factor, once for the family
  if (!sparse_analyze(f, 0, sym_))
    throw std::invalid_argument("sov_lp_solve_family: the sparse L D L' of the order-" + std::to_string(f.m) +
                                " normal matrix needs more than " + std::to_string(kMaxUpdates) +
                                " rank-1 update terms");
  // the trailing block -- the root clique of the elimination tree and the nearly dense columns
  // before it -- is factored and solved densely when that costs less than scheduling its terms;
  // one thread per (piece, LP): long items are cut into short pieces
  tail_ = sparse_dense_block(sym_, kSparseTermCost, kMinTail);
  const SparseSchedule S = sparse_schedule(sym_, tail_, kFamPiece);
  {
    const int T = tail_, mt = f.m - T;
    std::vector<int> off(std::max(1, T)), src, dst;
    for (int q = 0; q < T; ++q) off[q] = q * (T - 1) - q * (q - 1) / 2;
    for (int q = 0; q < T; ++q)
      for (int p = sym_.lp[mt + q]; p < sym_.lp[mt + q + 1]; ++p) {
        src.push_back(f.m + p);
        dst.push_back(off[q] + (sym_.li[p] - (mt + q) - 1));
      }
    tail_off_.put(off, st_);
    blk_src_.put(src, st_);
    blk_dst_.put(dst, st_);
    blk_n_ = static_cast<int>(src.size());
    ld_size_ = static_cast<size_t>(T) * (T > 0 ? T - 1 : 0) / 2;
  }
  pivot_ptr_.put(S.pivot_ptr, st_);
  pivot_col_.put(S.pivot_col, st_);
  row_ptr_.put(f.row_ptr, st_);
  col_idx_.put(f.col_idx, st_);
  rval_.put(f.rval, st_);
  col_ptr_.put(f.col_ptr, st_);
  row_idx_.put(f.row_idx, st_);
  cval_.put(f.val, st_);
  asm_target_.put(sym_.asm_target, st_);
  asm_ptr_.put(sym_.asm_ptr, st_);
  asm_col_.put(sym_.asm_col, st_);
  asm_w_.put(sym_.asm_w, st_);
  perm_.put(sym_.perm, st_);
  lvl_ptr_.put(sym_.lvl_ptr, st_);
  lvl_col_.put(sym_.lvl_col, st_);
  li_.put(sym_.li, st_);
  up_col_.put(S.up_col, st_);
  up_a_.put(S.up_a, st_);
  up_b_.put(S.up_b, st_);
  row_pos_.put(S.row_pos, st_);
  row_col_.put(S.row_col, st_);
  static_assert(sizeof(SparsePiece) == sizeof(int4) && sizeof(SparseCombine) == sizeof(int4), "piece layout");
  auto put4 = [&](Buf<int4>& b, const auto& v) {
    std::vector<int4> w(v.size());
    std::memcpy(w.data(), v.data(), sizeof(int4) * v.size());
    b.put(w, st_);
  };
  put4(fp_, S.factor.piece);
  put4(fc_, S.factor.comb);
  put4(lpc_, S.forward.piece);
  put4(lc_, S.forward.comb);
  put4(upc_, S.backward.piece);
  put4(uc_, S.backward.comb);
  fpl_.put(S.factor.piece_lvl, st_);
  fcl_.put(S.factor.comb_lvl, st_);
  lpl_.put(S.forward.piece_lvl, st_);
  lcl_.put(S.forward.comb_lvl, st_);
  upl_.put(S.backward.piece_lvl, st_);
  ucl_.put(S.backward.comb_lvl, st_);
  slots_ = std::max(1, std::max(S.factor_slots, S.solve_slots));
  SOV_CUDA(cudaStreamSynchronize(st_));  // host vectors above go out of scope
  // per-chunk storage at the full width
  const size_t W = kFamilyWidth, n = f.n, m = f.m;
  for (Buf<double>* v : {&c_, &x_, &s_, &dx_, &ds_, &dxa_, &dsa_, &rd_, &t_, &x0_, &s0_, &bx_, &bs_, &cx_, &cs_})
    v->alloc(n * W);
  for (Buf<double>* v : {&b_, &y_, &rp_, &z_, &y0_, &by_, &cy_, &diag_, &inv_d_, &work_}) v->alloc(m * W);
  bnorm_.alloc(W);
  cnorm_.alloc(W);
  part_.alloc(static_cast<size_t>(kFamBlocks) * kNv * W);
  part_rows_.alloc(static_cast<size_t>(kFamBlocks) * kNv * W);
  V_.alloc((m + sym_.li.size()) * W);
  Ld_.alloc(std::max<size_t>(1, ld_size_) * W);
  partial_.alloc(static_cast<size_t>(slots_) * W);
  sc_.alloc(W);
  step_.alloc(W);
  mask_.alloc(W);
  SOV_CUDA(cudaMallocHost(&hsc_, sizeof(FamScalars) * W));
  int dev = 0;
  SOV_CUDA(cudaGetDevice(&dev));
  SOV_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
  SOV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_factor_, k_fam_factor, kFamThreads, 0));
  SOV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_solve_, k_fam_solve, kFamThreads, 0));
  per_sm_factor_ = std::max(1, std::min(per_sm_factor_, 2));
  per_sm_solve_ = std::max(1, std::min(per_sm_solve_, 2));
  am_ = FamAssembly{asm_target_.p, asm_ptr_.p, asm_col_.p, asm_w_.p, static_cast<int>(sym_.asm_target.size())};
  sp_.m = f.m;
  sp_.levels = S.levels;
  sp_.tail = tail_;
  sp_.mt = f.m - tail_;
  sp_.tail_off = tail_off_.p;
  sp_.Ld = Ld_.p;
  sp_.blk_src = blk_src_.p;
  sp_.blk_dst = blk_dst_.p;
  sp_.blk_n = blk_n_;
  sp_.pivot_ptr = pivot_ptr_.p;
  sp_.pivot_col = pivot_col_.p;
  sp_.V = V_.p;
  sp_.diag = diag_.p;
  sp_.inv_d = inv_d_.p;
  sp_.work = work_.p;
  sp_.partial = partial_.p;
  sp_.perm = perm_.p;
  sp_.lvl_ptr = lvl_ptr_.p;
  sp_.lvl_col = lvl_col_.p;
  sp_.li = li_.p;
  sp_.fpiece = fp_.p;
  sp_.fcomb = fc_.p;
  sp_.lpiece = lpc_.p;
  sp_.lcomb = lc_.p;
  sp_.upiece = upc_.p;
  sp_.ucomb = uc_.p;
  sp_.fpiece_lvl = fpl_.p;
  sp_.fcomb_lvl = fcl_.p;
  sp_.lpiece_lvl = lpl_.p;
  sp_.lcomb_lvl = lcl_.p;
  sp_.upiece_lvl = upl_.p;
  sp_.ucomb_lvl = ucl_.p;
  sp_.up_col = up_col_.p;
  sp_.up_a = up_a_.p;
  sp_.up_b = up_b_.p;
  sp_.row_pos = row_pos_.p;
  sp_.row_col = row_col_.p;
  sp_.sc = sc_.p;
  sp_.drop_tol = 1e-13;
  dev_.m = f.m;
  dev_.n = f.n;
  dev_.row_ptr = row_ptr_.p;
  dev_.col_idx = col_idx_.p;
  dev_.col_ptr = col_ptr_.p;
  dev_.row_idx = row_idx_.p;
  dev_.rval = rval_.p;
  dev_.cval = cval_.p;
  dev_.b = b_.p;
  dev_.c = c_.p;
  dev_.bnorm = bnorm_.p;
  dev_.cnorm = cnorm_.p;
  dev_.x = x_.p;
  dev_.s = s_.p;
  dev_.y = y_.p;
  dev_.dx = dx_.p;
  dev_.ds = ds_.p;
  dev_.dxa = dxa_.p;
  dev_.dsa = dsa_.p;
  dev_.rd = rd_.p;
  dev_.rp = rp_.p;
  dev_.z = z_.p;
  dev_.t = t_.p;
  dev_.sc = sc_.p;
  dev_.step = step_.p;
  dev_.part = part_.p;
}

void Family::residuals() {
  const int W = dev_.W, bd = W * dev_.G;
  const size_t smem = sizeof(double) * kNv * bd;
  FamDev rows = dev_;
  rows.part = part_rows_.p;
  const int gr = grid_for(dev_.m), gc = grid_for(dev_.n);
  k_fam_res_rows<<<gr, bd, smem, st_>>>(rows);
  k_fam_res_cols<<<gc, bd, smem, st_>>>(dev_);
  k_fam_res_final<<<1, kFamilyWidth, 0, st_>>>(dev_, part_rows_.p, gr, gc);
  SOV_LAUNCH_CHECK();
}

void Family::assemble(bool ones) {
  SOV_CUDA(cudaMemsetAsync(V_.p, 0, sizeof(double) * (dev_.m + sym_.li.size()) * dev_.W, st_));
  const long long total = static_cast<long long>(am_.ntargets) * dev_.W;
  const int blocks = static_cast<int>(std::max(1LL, std::min(8LL * sms_, (total + 255) / 256)));
  k_fam_assemble<<<blocks, 256, 0, st_>>>(am_, dev_, sp_, ones ? 1 : 0);
  SOV_LAUNCH_CHECK();
}

void Family::factor() {
  FamSparse f = sp_;
  void* args[] = {&f};
  SOV_CUDA(cudaLaunchCooperativeKernel((const void*)k_fam_factor, dim3(sms_ * per_sm_factor_), dim3(kFamThreads), args,
                                       0, st_));
  if (tail_ > 0) {
    SOV_CUDA(cudaMemsetAsync(Ld_.p, 0, sizeof(double) * ld_size_ * sp_.W, st_));
    const long long total = static_cast<long long>(blk_n_) * sp_.W;
    k_tail_scatter<<<static_cast<int>(std::max(1LL, std::min(8LL * sms_, (total + 255) / 256))), 256, 0, st_>>>(sp_);
  }
  for (int j0 = 0; j0 < tail_; j0 += kPanel) {
    const int j1 = std::min(tail_, j0 + kPanel), W = sp_.W;
    k_tail_diag<<<1, (j1 - j0) * W, 0, st_>>>(sp_, j0, j1);
    if (j1 < tail_) {
      const long long rows = static_cast<long long>(tail_ - j1) * W;
      const long long n = tail_ - j1, nt = (n + 3) / 4, pairs = nt * (nt + 1) / 2 * W;
      k_tail_rows<<<static_cast<int>(std::max(1LL, std::min(8LL * sms_, (rows + 255) / 256))), 256, 0, st_>>>(sp_, j0, j1);
      k_tail_update<<<static_cast<int>(std::max(1LL, std::min(16LL * sms_, (pairs + 255) / 256))), 256, 0, st_>>>(sp_, j0,
                                                                                                            j1);
    }
  }
  SOV_LAUNCH_CHECK();
}

void Family::solve(double* z) {
  FamSparse f = sp_;
  void* args[] = {&f, &z};
  SOV_CUDA(cudaLaunchCooperativeKernel((const void*)k_fam_solve, dim3(sms_ * per_sm_solve_), dim3(kFamThreads), args, 0,
                                       st_));
}

void Family::copy(int entries, const int* mask_dev, double* dst, const double* src) {
  const long long total = static_cast<long long>(entries) * dev_.W;
  const int blocks = static_cast<int>(std::max(1LL, std::min(8LL * sms_, (total + 255) / 256)));
  k_fam_copy<<<blocks, 256, 0, st_>>>(entries, dev_.W, mask_dev, dst, src);
  SOV_LAUNCH_CHECK();
}

std::string Family::describe() const {
  char buf[256];
  std::snprintf(buf, sizeof buf,
                "sparse LDL^T on the GPU with %s ordering (order %d, nnz(L) = %lld, %d levels, dense trailing "
                "block of %d columns), one symbolic factor for the family, %d LPs per launch",
                sym_.ordering == SparseOrder::kNestedDissection ? "nested-dissection" : "minimum-degree", sym_.m,
                sym_.nnz_l, sp_.levels, tail_, dev_.W);
  return buf;
}

// a slot's failure flags cleared (a restart, or the next LP taking the slot)
__global__ void k_fam_clear_fail(FamScalars* sc, const int* mask, int W) {
  const int k = threadIdx.x;
  if (k < W && (!mask || mask[k])) {
    sc[k].fail = 0;
    sc[k].skipped = 0;
  }
}

void Family::solve_wave(const std::vector<int>& lps) {
  const int count = static_cast<int>(lps.size());
  const int W = std::min(kFamilyWidth, count);
  const StdForm& f0 = forms_[lps[0]];
  const int n = f0.n, m = f0.m;
  dev_.W = W;
  dev_.G = std::max(1, kFamThreads / W);
  dev_.tau = opts_[lps[0]].fraction_to_boundary;
  sp_.W = W;
  const auto t_start = std::chrono::steady_clock::now();
  const int bd = W * dev_.G, gn = grid_for(n);
  const size_t smem = sizeof(double) * kNv * bd;
  // ---- the wave's data on the device, one LP after another: b, c and the default starts ----
  Buf<double> bpool, cpool, x0p, y0p, s0p, stage;
  Buf<int> slot_dev, iota_dev;
  std::vector<double> bn(count), cn(count);
  {
    std::vector<double> hb(static_cast<size_t>(count) * m), hc(static_cast<size_t>(count) * n);
    for (int i = 0; i < count; ++i) {
      const StdForm& f = forms_[lps[i]];
      std::copy(f.b.begin(), f.b.end(), hb.begin() + static_cast<size_t>(i) * m);
      std::copy(f.c.begin(), f.c.end(), hc.begin() + static_cast<size_t>(i) * n);
      double bm = 0.0, cm = 0.0;
      for (double v : f.b) bm = std::max(bm, std::abs(v));
      for (double v : f.c) cm = std::max(cm, std::abs(v));
      bn[i] = std::max(1.0, bm);  // max(1, max |.|) of the scaled problem
      cn[i] = std::max(1.0, cm);
    }
    bpool.put(hb, st_);
    cpool.put(hc, st_);
    SOV_CUDA(cudaStreamSynchronize(st_));
  }
  x0p.alloc(static_cast<size_t>(count) * n);
  s0p.alloc(static_cast<size_t>(count) * n);
  y0p.alloc(static_cast<size_t>(count) * m);
  stage.alloc(static_cast<size_t>(W) * (2 * n + m));
  slot_dev.alloc(W);
  {
    std::vector<int> iota(W);
    for (int k = 0; k < W; ++k) iota[k] = k;
    iota_dev.put(iota, st_);
  }
  // slot norms, held on the host and uploaded whole when they change
  std::vector<double> bnorm_h(W, 1.0), cnorm_h(W, 1.0);
  auto put_norms = [&]() {
    SOV_CUDA(cudaMemcpyAsync(bnorm_.p, bnorm_h.data(), sizeof(double) * W, cudaMemcpyHostToDevice, st_));
    SOV_CUDA(cudaMemcpyAsync(cnorm_.p, cnorm_h.data(), sizeof(double) * W, cudaMemcpyHostToDevice, st_));
  };
  std::vector<int> hmask(W);
  auto put_mask = [&]() {
    SOV_CUDA(cudaMemcpyAsync(mask_.p, hmask.data(), sizeof(int) * W, cudaMemcpyHostToDevice, st_));
  };
  auto read_scalars = [&]() {
    SOV_CUDA(cudaMemcpyAsync(hsc_, sc_.p, sizeof(FamScalars) * W, cudaMemcpyDeviceToHost, st_));
    SOV_CUDA(cudaStreamSynchronize(st_));
  };
  // slots of unused width hold finite values: every per-LP pass reads its own slot only
  k_fill<<<sms_, 256, 0, st_>>>(x_.p, static_cast<long long>(n) * W, 1.0);
  k_fill<<<sms_, 256, 0, st_>>>(s_.p, static_cast<long long>(n) * W, 1.0);
  k_fill<<<sms_, 256, 0, st_>>>(y_.p, static_cast<long long>(m) * W, 0.0);
  SOV_CUDA(cudaMemsetAsync(sc_.p, 0, sizeof(FamScalars) * W, st_));
  // supplied starts: a host copy of those that are kept, uploaded when the LP takes a slot
  std::vector<char> warm_used(count, 0);
  auto warm_of = [&](int i) {
    const sov_options& o = opts_[lps[i]];
    return o.warm_x && o.warm_y && o.warm_s;
  };
  // ---- default starts (Engine::run's default_start): A A' dy = b - A 1 for W LPs at a time; the
  // supplied starts judged against them by the single engine's safeguard ----
  for (int g0 = 0; g0 < count; g0 += W) {
    const int G = std::min(W, count - g0);
    put_slots(b_.p, m, iota_dev.p, bpool.p + static_cast<size_t>(g0) * m, G);
    put_slots(c_.p, n, iota_dev.p, cpool.p + static_cast<size_t>(g0) * n, G);
    for (int k = 0; k < G; ++k) {
      bnorm_h[k] = bn[g0 + k];
      cnorm_h[k] = cn[g0 + k];
    }
    put_norms();
    SOV_CUDA(cudaMemsetAsync(sc_.p, 0, sizeof(FamScalars) * W, st_));
    assemble(true);
    factor();
    k_fam_start_rhs<<<grid_for(m), bd, 0, st_>>>(dev_);
    solve(z_.p);
    k_fam_start_point<<<grid_for(std::max(n, m)), bd, 0, st_>>>(dev_, x0_.p, y0_.p, s0_.p);
    SOV_LAUNCH_CHECK();
    get_slots(x0p.p + static_cast<size_t>(g0) * n, n, iota_dev.p, x0_.p, G);
    get_slots(s0p.p + static_cast<size_t>(g0) * n, n, iota_dev.p, s0_.p, G);
    get_slots(y0p.p + static_cast<size_t>(g0) * m, m, iota_dev.p, y0_.p, G);
    bool any_warm = false;
    for (int k = 0; k < G; ++k) any_warm |= warm_of(g0 + k);
    if (!any_warm) continue;
    SOV_CUDA(cudaMemcpyAsync(x_.p, x0_.p, sizeof(double) * n * W, cudaMemcpyDeviceToDevice, st_));
    SOV_CUDA(cudaMemcpyAsync(s_.p, s0_.p, sizeof(double) * n * W, cudaMemcpyDeviceToDevice, st_));
    SOV_CUDA(cudaMemcpyAsync(y_.p, y0_.p, sizeof(double) * m * W, cudaMemcpyDeviceToDevice, st_));
    residuals();
    read_scalars();
    std::vector<double> dmetric(G), dmu(G);
    for (int k = 0; k < G; ++k) {
      dmetric[k] = hsc_[k].metric;
      dmu[k] = hsc_[k].mu;
    }
    // the supplied starts into their slots: x | s | y of each, staged contiguously
    std::vector<int> ws;
    std::vector<double> hx, hs, hy;
    for (int k = 0; k < G; ++k) {
      if (!warm_of(g0 + k)) continue;
      const sov_options& o = opts_[lps[g0 + k]];
      ws.push_back(k);
      hx.insert(hx.end(), o.warm_x, o.warm_x + n);
      hs.insert(hs.end(), o.warm_s, o.warm_s + n);
      hy.insert(hy.end(), o.warm_y, o.warm_y + m);
    }
    const int nw = static_cast<int>(ws.size());
    SOV_CUDA(cudaMemcpyAsync(slot_dev.p, ws.data(), sizeof(int) * nw, cudaMemcpyHostToDevice, st_));
    double* sx = stage.p;
    double* ss = sx + static_cast<size_t>(nw) * n;
    double* sy = ss + static_cast<size_t>(nw) * n;
    SOV_CUDA(cudaMemcpyAsync(sx, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice, st_));
    SOV_CUDA(cudaMemcpyAsync(ss, hs.data(), sizeof(double) * hs.size(), cudaMemcpyHostToDevice, st_));
    SOV_CUDA(cudaMemcpyAsync(sy, hy.data(), sizeof(double) * hy.size(), cudaMemcpyHostToDevice, st_));
    put_slots(x_.p, n, slot_dev.p, sx, nw);
    put_slots(s_.p, n, slot_dev.p, ss, nw);
    put_slots(y_.p, m, slot_dev.p, sy, nw);
    residuals();
    read_scalars();
    for (int k : ws) {
      const FamScalars& sc = hsc_[k];
      warm_used[g0 + k] = std::isfinite(sc.metric) && std::isfinite(sc.mu) && sc.metric <= 10.0 * dmetric[k] &&
                          sc.mu <= dmu[k];
    }
  }
  // ---- the iteration loop: W slots, each running one LP through Engine::run's decisions; a slot
  // whose LP has finished takes the next LP of the wave ----
  std::vector<int> slot_lp(W, -1), it_of(W, 0);
  std::vector<LpState> L(W);
  int next = 0;
  std::vector<int> hstep(W), hbest(W), hrestart(W), hcap(W);
  const char* fail_text =
      "IPM stopped because the affine predictor factorization failed; the best iterate is returned with optimality "
      "unproven.";
  // results of finished LPs: their vectors gathered from the slots, then published on the host
  std::vector<double> hres;
  Buf<double> out;
  out.alloc(static_cast<size_t>(W) * 3 * (2 * n + m));
  auto retire = [&](const std::vector<int>& done, const std::vector<char>& from_best) {
    const int F = static_cast<int>(done.size());
    if (!F) return;
    bool any_cap = false;
    for (int k : done) any_cap |= L[k].captured;
    const size_t per = static_cast<size_t>(2 * n + m) * (any_cap ? 3 : 2);
    SOV_CUDA(cudaMemcpyAsync(slot_dev.p, done.data(), sizeof(int) * F, cudaMemcpyHostToDevice, st_));
    // layout per block: current x (F n) | s (F n) | y (F m), then the best ones, then captured
    const double* src[3][3] = {{x_.p, s_.p, y_.p}, {bx_.p, bs_.p, by_.p}, {cx_.p, cs_.p, cy_.p}};
    const size_t blk = static_cast<size_t>(2 * n + m) * F;
    for (int b = 0; b < (any_cap ? 3 : 2); ++b) {
      double* o = out.p + b * blk;
      get_slots(o, n, slot_dev.p, src[b][0], F);
      get_slots(o + static_cast<size_t>(F) * n, n, slot_dev.p, src[b][1], F);
      get_slots(o + static_cast<size_t>(2 * F) * n, m, slot_dev.p, src[b][2], F);
    }
    hres.resize(per * F);
    SOV_CUDA(cudaMemcpyAsync(hres.data(), out.p, sizeof(double) * hres.size(), cudaMemcpyDeviceToHost, st_));
    SOV_CUDA(cudaStreamSynchronize(st_));
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_start).count();
    for (int i = 0; i < F; ++i) {
      const int k = done[i];
      const double* o = hres.data() + (from_best[i] ? blk : 0);
      const double* c = any_cap && L[k].captured ? hres.data() + 2 * blk : nullptr;
      publish(L[k], o + static_cast<size_t>(i) * n, o + static_cast<size_t>(2 * F) * n + static_cast<size_t>(i) * m,
              o + static_cast<size_t>(F) * n + static_cast<size_t>(i) * n,
              c ? c + static_cast<size_t>(i) * n : nullptr,
              c ? c + static_cast<size_t>(2 * F) * n + static_cast<size_t>(i) * m : nullptr,
              c ? c + static_cast<size_t>(F) * n + static_cast<size_t>(i) * n : nullptr, secs);
      slot_lp[k] = -1;
    }
  };
  // free slots take the next LPs: data, start (default or the kept supplied one), bookkeeping
  auto refill = [&]() {
    std::vector<int> fs;
    for (int k = 0; k < W && next + static_cast<int>(fs.size()) < count; ++k)
      if (slot_lp[k] < 0) fs.push_back(k);
    const int F = static_cast<int>(fs.size());
    if (!F) return;
    const int c0 = next;
    next += F;
    SOV_CUDA(cudaMemcpyAsync(slot_dev.p, fs.data(), sizeof(int) * F, cudaMemcpyHostToDevice, st_));
    put_slots(b_.p, m, slot_dev.p, bpool.p + static_cast<size_t>(c0) * m, F);
    put_slots(c_.p, n, slot_dev.p, cpool.p + static_cast<size_t>(c0) * n, F);
    put_slots(x_.p, n, slot_dev.p, x0p.p + static_cast<size_t>(c0) * n, F);
    put_slots(s_.p, n, slot_dev.p, s0p.p + static_cast<size_t>(c0) * n, F);
    put_slots(y_.p, m, slot_dev.p, y0p.p + static_cast<size_t>(c0) * m, F);
    std::vector<int> ws;
    std::vector<double> hx, hs, hy;
    std::fill(hmask.begin(), hmask.end(), 0);
    for (int i = 0; i < F; ++i) {
      const int k = fs[i], w = c0 + i;
      hmask[k] = 1;
      slot_lp[k] = w;
      it_of[k] = 0;
      bnorm_h[k] = bn[w];
      cnorm_h[k] = cn[w];
      LpState& l = L[k];
      l = LpState{};
      l.idx = lps[w];
      l.o = opts_[lps[w]];
      l.factorizations = 1;  // the start system's
      l.warm_used = warm_used[w] != 0;
      const StdForm& f = forms_[lps[w]];
      sov_diagnostics& dg = l.dg;
      dg.scaling_applied = f.scaling_applied;
      dg.coefficient_min_abs_before = f.coef_min_before;
      dg.coefficient_max_abs_before = f.coef_max_before;
      dg.coefficient_min_abs_after = f.coef_min_after;
      dg.coefficient_max_abs_after = f.coef_max_after;
      dg.stall_iteration = -1;
      dg.warm_start_used = l.warm_used ? 1 : 0;
      if (l.warm_used) {
        ws.push_back(k);
        hx.insert(hx.end(), l.o.warm_x, l.o.warm_x + n);
        hs.insert(hs.end(), l.o.warm_s, l.o.warm_s + n);
        hy.insert(hy.end(), l.o.warm_y, l.o.warm_y + m);
      }
    }
    if (!ws.empty()) {
      const int nw = static_cast<int>(ws.size());
      Buf<int> wslots;
      wslots.put(ws, st_);
      double* sx = stage.p;
      double* ss = sx + static_cast<size_t>(nw) * n;
      double* sy = ss + static_cast<size_t>(nw) * n;
      SOV_CUDA(cudaMemcpyAsync(sx, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(ss, hs.data(), sizeof(double) * hs.size(), cudaMemcpyHostToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(sy, hy.data(), sizeof(double) * hy.size(), cudaMemcpyHostToDevice, st_));
      put_slots(x_.p, n, wslots.p, sx, nw);
      put_slots(s_.p, n, wslots.p, ss, nw);
      put_slots(y_.p, m, wslots.p, sy, nw);
      SOV_CUDA(cudaStreamSynchronize(st_));  // wslots goes out of scope
    }
    put_norms();
    put_mask();
    copy(n, mask_.p, bx_.p, x_.p);
    copy(n, mask_.p, bs_.p, s_.p);
    copy(m, mask_.p, by_.p, y_.p);
    k_fam_clear_fail<<<1, kFamilyWidth, 0, st_>>>(sc_.p, mask_.p, W);
  };
  for (;;) {
    refill();
    bool any_active = false, any_cap = false;
    for (int k = 0; k < W; ++k) {
      const bool act = slot_lp[k] >= 0;
      hcap[k] = act && L[k].o.ipm_iterate_at == it_of[k] + 1;
      any_cap |= hcap[k] != 0;
      if (hcap[k]) L[k].captured = true;
      any_active |= act;
    }
    if (!any_active) break;
    if (any_cap) {
      hmask = hcap;
      put_mask();
      copy(n, mask_.p, cx_.p, x_.p);
      copy(n, mask_.p, cs_.p, s_.p);
      copy(m, mask_.p, cy_.p, y_.p);
    }
    residuals();
    read_scalars();
    bool any_step = false, any_best = false;
    std::vector<int> done, restarts;
    std::vector<char> from_best;
    for (int k = 0; k < W; ++k) {
      hstep[k] = hbest[k] = hrestart[k] = 0;
      if (slot_lp[k] < 0) continue;
      LpState& l = L[k];
      const int it = it_of[k]++;  // Engine::run's iteration counter for this LP
      const FamScalars s = hsc_[k];
      sov_diagnostics& dg = l.dg;
      if (it >= l.o.max_iterations) {  // the loop of this LP has ended without convergence
        char buf[512];
        std::snprintf(buf, sizeof buf,
                      "IPM stopped after %d iterations without meeting tolerance; returning best iterate from %d as a "
                      "lower-accuracy candidate. Relative duality gap = %g (tolerance %g), primal residual = %g, dual "
                      "residual = %g. Optimality is not proven.",
                      l.o.max_iterations, l.best_it, l.best_gap, l.o.optimality_tol, l.best_p, l.best_d);
        l.msg = buf;
        done.push_back(k);
        from_best.push_back(1);
        continue;
      }
      if (it > 0) {
        const int prev = it - 1;
        const bool prev_sample = prev < 8 || prev % 10 == 0 || prev + 1 == l.o.max_iterations;
        if (prev_sample && dg.step_history_len < SOV_HISTORY_MAX) {
          dg.primal_step_history[dg.step_history_len] = s.alpha_p;
          dg.dual_step_history[dg.step_history_len] = s.alpha_d;
          dg.step_history_len++;
        }
        if (dg.stall_iteration == prev + 1) {
          dg.stall_primal_step = s.alpha_p;
          dg.stall_dual_step = s.alpha_d;
        }
      }
      if (s.fail || s.skipped) {
        l.msg = fail_text;
        done.push_back(k);
        from_best.push_back(1);
        continue;
      }
      if (s.metric < l.best_metric) {
        l.best_metric = s.metric;
        hbest[k] = 1;
        any_best = true;
        l.best_gap = s.gap;
        l.best_p = s.p_res;
        l.best_d = s.d_res;
        l.best_it = it + 1;
        l.stale = 0;
      } else {
        ++l.stale;
      }
      const bool sample = it < 8 || it % 10 == 0 || it + 1 == l.o.max_iterations;
      if (sample && dg.history_len < SOV_HISTORY_MAX) {
        dg.history_iterations[dg.history_len] = it + 1;
        dg.objective_history[dg.history_len] = s.cx;
        dg.gap_history[dg.history_len] = s.gap;
        dg.mu_history[dg.history_len] = s.mu;
        dg.history_len++;
      }
      if (s.gap < l.best_gap) {
        l.best_gap = s.gap;
        l.stale = 0;
      } else if (l.stale >= 8 && dg.stall_iteration < 0) {
        dg.stall_iteration = it + 1;
        dg.stall_gap = s.gap;
        dg.stall_mu = s.mu;
      }
      if (s.p_res < l.o.feasibility_tol && s.d_res < l.o.feasibility_tol && s.gap < l.o.optimality_tol) {
        l.optimal = true;
        l.its = it + 1;
        l.gap = s.gap;
        l.p_res = s.p_res;
        l.d_res = s.d_res;
        done.push_back(k);
        from_best.push_back(0);
        continue;
      }
      if (l.warm_used && it + 1 == kWarmGiveUp) {  // the supplied start is abandoned once
        l.warm_used = false;
        dg.warm_start_used = 0;
        restarts.push_back(k);
        l.best_metric = l.best_gap = l.best_p = l.best_d = INFINITY;
        l.best_it = 0;
        l.stale = 0;
        l.factorizations++;
        continue;
      }
      hstep[k] = 1;
      any_step = true;
    }
    if (any_best) {
      hmask = hbest;
      put_mask();
      copy(n, mask_.p, bx_.p, x_.p);
      copy(n, mask_.p, bs_.p, s_.p);
      copy(m, mask_.p, by_.p, y_.p);
    }
    for (int k : restarts) {  // back to this LP's default start
      const int w = slot_lp[k];
      SOV_CUDA(cudaMemcpyAsync(slot_dev.p, &k, sizeof(int), cudaMemcpyHostToDevice, st_));
      put_slots(x_.p, n, slot_dev.p, x0p.p + static_cast<size_t>(w) * n, 1);
      put_slots(s_.p, n, slot_dev.p, s0p.p + static_cast<size_t>(w) * n, 1);
      put_slots(y_.p, m, slot_dev.p, y0p.p + static_cast<size_t>(w) * m, 1);
      std::fill(hmask.begin(), hmask.end(), 0);
      hmask[k] = 1;
      put_mask();
      k_fam_clear_fail<<<1, kFamilyWidth, 0, st_>>>(sc_.p, mask_.p, W);
    }
    retire(done, from_best);
    if (!any_step) continue;
    SOV_CUDA(cudaMemcpyAsync(step_.p, hstep.data(), sizeof(int) * W, cudaMemcpyHostToDevice, st_));
    assemble(false);
    factor();
    for (int pass = 0; pass < 2; ++pass) {
      k_fam_newton_tmp<<<gn, bd, 0, st_>>>(dev_, pass);
      k_fam_newton_rhs<<<grid_for(m), bd, 0, st_>>>(dev_);
      solve(z_.p);
      k_fam_direction<<<gn, bd, smem, st_>>>(dev_, pass);
      k_fam_direction_final<<<1, kFamilyWidth, 0, st_>>>(dev_, pass, gn);
      if (pass == 0) {
        k_fam_mu_aff<<<gn, bd, smem, st_>>>(dev_);
        k_fam_mu_final<<<1, kFamilyWidth, 0, st_>>>(dev_, gn);
      }
    }
    k_fam_update<<<grid_for(std::max(n, m)), bd, 0, st_>>>(dev_);
    SOV_LAUNCH_CHECK();
    for (int k = 0; k < W; ++k) L[k].factorizations += hstep[k];
  }
  SOV_CUDA(cudaStreamSynchronize(st_));
}

void Family::publish(LpState& l, const double* x, const double* y, const double* s, const double* cx,
                     const double* cy, const double* cs, double seconds) {
  const StdForm& f = forms_[l.idx];
  const sov_model& model = models_[l.idx];
  sov_result* r = &results_[l.idx];
  const int n = f.n, m = f.m;
  r->n_ipm = n;
  r->m_ipm = m;
  if (l.optimal) {
    r->status = SOV_OPTIMAL;
    r->iterations = l.its;
    r->duality_gap = l.gap;
    r->primal_residual = l.p_res;
    r->dual_residual = l.d_res;
    l.msg = "Optimal solution found by primal-dual interior-point (Mehrotra). Normal equations: " + describe() + ".";
  } else {
    r->status = l.best_p <= l.o.feasibility_tol ? SOV_FEASIBLE : SOV_NUMERICAL_ERROR;
    r->iterations = l.best_it;
    r->duality_gap = l.best_gap;
    r->primal_residual = l.best_p;
    r->dual_residual = l.best_d;
  }
  r->has_objective_value = 1;
  double obj = model.obj_constant;
  for (int j = 0; j < f.n_struct; ++j) {
    const double v = f.shift[j] + f.col_scale[j] * x[j];
    if (r->primal) r->primal[j] = v;
    if (r->dual_col) r->dual_col[j] = s[j] / f.col_scale[j];
    obj += (model.obj ? model.obj[j] : 0.0) * v;
  }
  if (r->dual_row)
    for (int i = 0; i < f.m0; ++i) r->dual_row[i] = f.row_scale[i] * y[i];
  const bool cap = l.captured && cx;
  if (r->ipm_x) std::copy(cap ? cx : x, (cap ? cx : x) + n, r->ipm_x);
  if (r->ipm_s) std::copy(cap ? cs : s, (cap ? cs : s) + n, r->ipm_s);
  if (r->ipm_y) std::copy(cap ? cy : y, (cap ? cy : y) + m, r->ipm_y);
  r->objective_value = obj;
  r->solve_seconds = seconds;
  std::snprintf(r->message, sizeof(r->message), "%s", l.msg.c_str());
  if (r->diagnostics) {
    l.dg.refactorizations = l.factorizations;
    *r->diagnostics = l.dg;
  }
}

void Family::put_slots(double* dst, int len, const int* slots, const double* src, int count) {
  const long long total = static_cast<long long>(count) * len;
  if (total <= 0) return;
  k_slot_put<<<static_cast<int>(std::max(1LL, std::min(8LL * sms_, (total + 255) / 256))), 256, 0, st_>>>(
      dst, len, dev_.W, slots, src, count);
  SOV_LAUNCH_CHECK();
}

void Family::get_slots(double* dst, int len, const int* slots, const double* src, int count) {
  const long long total = static_cast<long long>(count) * len;
  if (total <= 0) return;
  k_slot_get<<<static_cast<int>(std::max(1LL, std::min(8LL * sms_, (total + 255) / 256))), 256, 0, st_>>>(
      dst, len, dev_.W, slots, src, count);
  SOV_LAUNCH_CHECK();
}

}  // namespace

int solve_family(int count, const sov_model* models, const sov_options* opt, int opt_stride, sov_result* results) {
  if (count <= 0) return SOV_OK;
  for (int k = 0; k < count; ++k) {
    results[k].status = SOV_ERROR;
    results[k].iterations = 0;
    results[k].has_objective_value = 0;
    results[k].message[0] = '\0';
  }
  Family fam(count, models, opt, opt_stride, results);
  return fam.run();
}

}  // namespace sov
