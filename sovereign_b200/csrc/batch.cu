// batch.cu -- batched persistent interior-point solver: thousands of small LPs in one launch.
//
// One CTA owns one LP at a time and runs the whole Mehrotra predictor-corrector loop of
// solve_ipm (solver/lp/src/interior_point.cpp:454-740) for it without returning to the host:
// CTAs pull LP indices from a device counter (largest first), so uneven sizes balance across
// the 148 SMs. The normal matrix of an LP (order m <= 128; lower triangle packed by rows, 66 KB at
// m = 128, so up to three LPs share an SM) lives in shared memory and is factored there as L D L'
// with the reference's dependent-row rule; n-vectors stay in global memory, where
// the working set of the resident CTAs fits in the 126 MB L2. Size buckets (by m) get their own
// launch with a shared-memory footprint and thread count chosen per bucket by the autotuner; the
// bucket launches of a batch run concurrently on forked streams, captured once in a CUDA graph.
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <numeric>
#include <sstream>
#include <thread>
#include <vector>

#include "batch.hpp"
#include "common.cuh"
#include "dense.cuh"
#include "engine.hpp"
#include "stdform.hpp"

namespace sov {

constexpr int kBatchMaxRows = 128;
constexpr int kWarmGiveUp = 40;  // iterations a supplied start gets before the Mehrotra restart

// offset of row i of a row-packed lower triangle
__host__ __device__ constexpr int tri(int i) { return i * (i + 1) / 2; }

struct LpMeta {
  int m, n, nnz, n_struct;  // IPM rows / columns / entries; the model's columns
  int max_iter, m0;         // the model's rows
  int scale_mode, pad0;     // scaling: 0 none, 1 on the device (k_batch_scale), 2 by the host
  long long a_off, cp_off, rp_off, mv_off, nv_off;
  long long w_off;  // caller's start [x (n) | y (m) | s (n)] in `warm`, or -1
  long long p_off;  // published [cs*x (n_struct) | s/cs (n_struct) | rs*y (m0)] in `pout`
  double bnorm, cnorm, ftol, otol, tau;
};

struct LpOut {
  int status, iterations, best_it, use_best;
  int drops, fail, warm_used, pad1;
  double gap, p_res, d_res, cx;
};

struct BatchDev {
  const LpMeta* meta;
  const int* order;
  int count;
  int* next;
  const int* col_ptr;
  const int* row_idx;
  const double* cval;
  const int* row_ptr;
  const int* col_idx;
  const double* rval;
  // per IPM column j (at nv_off + j): its first two entries inline -- rows (r0, r1), the column's
  // entry range [pb, pe) -- and their values (a0, a1), missing entries as row 0 with value 0; so
  // a column pass reads a column with two independent 16-byte loads instead of col_ptr first
  const int4* crec;
  const double2* cval2;
  const double* b;
  const double* c;
  const double* warm;
  double *x, *s, *dx, *ds, *dxa, *dsa, *rd, *bx, *bs;
  double *y, *by;
  LpOut* out;
};

namespace {

struct CtaScalars {
  double v[16];
  int flag[4];
};

// scalar slots
enum : int {
  S_MU = 0, S_PRES, S_DRES, S_GAP, S_METRIC, S_CX, S_APAFF, S_ADAFF, S_SIGMA, S_AP, S_AD, S_BEST
};

template <int NT>
__device__ __forceinline__ void cta_reduce4(double (&v)[4], const int (&ops)[4], double* red) {
  block_reduce<4>(v, ops, red);
}

template <int NT>
__device__ void solve_lp(const BatchDev& bd, const LpMeta& mt, int lp, double* sm, int mmax, double* red,
                         CtaScalars& cs) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int NW = NT / 32;
  const int m = mt.m, n = mt.n;
  // M: lower triangle, packed by rows (row i at tri(i)); then six m-vectors
  double* M = sm;
  double* vy = sm + tri(mmax + 1);
  double* vrp = vy + mmax;
  double* vz = vrp + mmax;
  double* vacc = vz + mmax;
  double* vdiag = vacc + mmax;
  double* vinv = vdiag + mmax;
  int* srp = reinterpret_cast<int*>(vinv + mmax);  // the row pointers (m + 1), read by every row pass

  const int* ri = bd.row_idx + mt.a_off;
  const double* cv = bd.cval + mt.a_off;
  const int* rpp = bd.row_ptr + mt.rp_off;
  const int* ci = bd.col_idx + mt.a_off;
  const double* rv = bd.rval + mt.a_off;
  const int4* crc = bd.crec + mt.nv_off;
  const double2* cv2 = bd.cval2 + mt.nv_off;
  const double* b = bd.b + mt.mv_off;
  const double* c = bd.c + mt.nv_off;
  double* x = bd.x + mt.nv_off;
  double* s = bd.s + mt.nv_off;
  double* dx = bd.dx + mt.nv_off;
  double* ds = bd.ds + mt.nv_off;
  double* dxa = bd.dxa + mt.nv_off;
  double* dsa = bd.dsa + mt.nv_off;
  double* rd = bd.rd + mt.nv_off;
  double* bx = bd.bx + mt.nv_off;
  double* bs = bd.bs + mt.nv_off;
  double* gy = bd.y + mt.mv_off;
  double* gby = bd.by + mt.mv_off;
  int drops = 0, fail = 0;

  // ---- normal matrix M = A diag(d) A' + 1e-12 I, assembled inside the residual passes ----
  // Off-diagonal entries come from the column pass: thread per column j, one shared-memory atomic
  // per pair of entries, (a_hj d_j) a_lj into M[h][l] (h > l). When no two rows share more than
  // one column (transportation LPs) each entry receives one term, so the order does not matter.
  // Diagonal entries come from the row pass as a warp sum of (a_ik a_ik) d_k over row i.
  // M is cleared by the pass before (start-up, or the update of the previous iteration).
  auto offdiag = [&](int pb, int pe, double dj) {
    for (int qa = pb; qa < pe; ++qa) {
      const int ra = ri[qa];
      const double va = cv[qa] * dj;
      for (int qb = pb; qb < pe; ++qb) {
        const int rb = ri[qb];
        if (rb < ra) atomicAdd(M + tri(ra) + rb, va * cv[qb]);
      }
    }
  };

  // the same from a column record: a column of two entries adds its one term straight from the
  // record (the product and the target of the loop above), longer columns take the loop
  auto offdiag_rec = [&](const int4 rc, const double2 av, double dj) {
    const int len = rc.w - rc.z;
    if (len == 2) {
      if (rc.y > rc.x) atomicAdd(M + tri(rc.y) + rc.x, (av.y * dj) * av.x);
      else if (rc.x > rc.y) atomicAdd(M + tri(rc.x) + rc.y, (av.x * dj) * av.y);
    } else if (len > 2) {
      offdiag(rc.z, rc.w, dj);
    }
  };

  // Row pass, RW rows per warp (all their gathers in flight), lanes over the row's entries:
  //  mode 0 (start):     z = b - A 1,                diag M_ii = sum a_ik^2 + 1e-12
  //  mode 1 (iteration): rp = b - A x, z = rp + A t,  diag M_ii = sum a_ik^2 d_k + 1e-12
  //  mode 2 (corrector): z = rp + A t with t = tv - smu dv (tv = t0, dv = w of the predictor pass)
  // Returns this thread's share of max |rp_i| (mode 1).
  constexpr int RW = 3;
  auto row_pass = [&](const int mode, const double* dv, const double* tv, double smu = 0.0) {
    double rpm = 0.0;
    for (int i0 = warp; i0 < m; i0 += RW * NW) {
      int rows[RW], pb[RW], pe[RW];
      double g0[RW], g1[RW], g2[RW];
      int len = 0;
#pragma unroll
      for (int h = 0; h < RW; ++h) {
        rows[h] = i0 + h * NW;
        pb[h] = rows[h] < m ? srp[rows[h]] : 0;
        pe[h] = rows[h] < m ? srp[rows[h] + 1] : 0;
        len = max(len, pe[h] - pb[h]);
        g0[h] = g1[h] = g2[h] = 0.0;
      }
      for (int o = lane; o < len; o += 32) {
#pragma unroll
        for (int h = 0; h < RW; ++h) {
          const int p = pb[h] + o;
          if (p < pe[h]) {
            const double a = rv[p];
            if (mode == 0) {
              g0[h] += a;
              g1[h] += a * a;
            } else {
              const int k = ci[p];
              if (mode == 1) {
                g0[h] += a * x[k];
                g1[h] += a * a * dv[k];
                g2[h] += a * tv[k];
              } else {
                g2[h] += a * (tv[k] - smu * dv[k]);
              }
            }
          }
        }
      }
#pragma unroll
      for (int h = 0; h < RW; ++h) {
        const double s0 = mode != 2 ? warp_sum(g0[h]) : 0.0;
        const double s1 = mode != 2 ? warp_sum(g1[h]) : 0.0;
        const double s2 = mode != 0 ? warp_sum(g2[h]) : 0.0;
        const int i = rows[h];
        if (i >= m) continue;
        if (mode == 2) {
          if (lane == 0) vz[i] = vrp[i] + s2;
          continue;
        }
        const double r = b[i] - s0;
        if (mode == 1) rpm = fmax(rpm, fabs(r));
        if (lane == 0) {
          M[tri(i) + i] = s1 + 1e-12;
          vdiag[i] = s1 + 1e-12;
          const double rhs = mode == 1 ? r + s2 : r;
          if (mode == 1) vrp[i] = r;
          vz[i] = rhs;
          M[tri(m) + i] = rhs;  // the augmented row of the factorization that follows
        }
      }
    }
    return rpm;
  };

  // ---- in-place L D L' (L~ = L D kept unscaled below the diagonal; vinv = 1/D) ----
  // Blocked right-looking over panels of KB columns, three barriers per panel:
  //  (1) warp 0 factors the KB x KB diagonal block, lane = row, one column at a time;
  //  (2) one thread per row below the block runs the same column recurrence on its KB panel
  //      entries held in registers;
  //  (3) the trailing lower triangle takes the panel's rank-KB update in 4 x 4 register tiles
  //      (8 shared loads per 16 FMAs instead of 3 shared accesses per FMA).
  // Every entry sees the same operations in the same order as the column-at-a-time algorithm
  // (M[i][j] -= (M[i][k] / D_k) * M[j][k] for k = 0, 1, ...), so the factor is bit-identical to it.
  // With `augmented`, row m holds a right-hand side r: it takes every column's update like any row
  // below the panels, which is the forward substitution, so afterwards M[m][k] = (L^-1 r)_k and
  // only the backward substitution is left for that right-hand side.
  // vdiag[k] (the assembled diagonal, the reference for the dependent-row test) is overwritten
  // with the pivot outcome of column k once it has been used: 0 kept, 1 dropped, 2 not finite.
  auto factor = [&](bool augmented) {
    constexpr int KB = 8;
    const int mr = augmented ? m + 1 : m;  // rows factored: row m carries a right-hand side
    for (int k0 = 0; k0 < m; k0 += KB) {
      const int k1 = min(k0 + KB, m);
      if (warp == 0) {
        for (int k = k0; k < k1; ++k) {
          const double p = M[tri(k) + k];
          const double dref = vdiag[k];
          // 2: not finite, 1: dependent row (sparse_ldlt.cpp:167-173), 0: kept; no branches
          const double code = !(fabs(p) <= DBL_MAX) ? 2.0 : (p <= 1e-13 * fabs(dref) ? 1.0 : 0.0);
          const double inv = 1.0 / (code != 0.0 ? 1e128 : p);
          const int i = k + 1 + lane;
          if (i < k1) {
            const double lik = M[tri(i) + k] * inv;
            double* Mi = M + tri(i);
            for (int j = k + 1; j <= i; ++j) Mi[j] -= lik * M[tri(j) + k];
          }
          __syncwarp();
          if (lane == 0) {
            vinv[k] = inv;
            vdiag[k] = code;
          }
        }
      }
      __syncthreads();
      for (int k = k0; k < k1; ++k) {
        const double code = vdiag[k];
        if (code == 1.0) ++drops;
        if (code == 2.0) fail = 1;
      }
      for (int i = k1 + tid; i < mr; i += NT) {
        double r[KB];
        double* Mi = M + tri(i) + k0;
#pragma unroll
        for (int a = 0; a < KB; ++a) r[a] = k0 + a < k1 ? Mi[a] : 0.0;
#pragma unroll
        for (int a = 0; a < KB; ++a) {
          if (k0 + a < k1) {
            const double l = r[a] * vinv[k0 + a];
#pragma unroll
            for (int c = a + 1; c < KB; ++c)
              if (k0 + c < k1) r[c] -= l * M[tri(k0 + c) + k0 + a];
          }
        }
#pragma unroll
        for (int a = 0; a < KB; ++a)
          if (k0 + a < k1) Mi[a] = r[a];
      }
      __syncthreads();
      const int tt = (mr - k1 + 3) >> 2;
      const int ntiles = tt * (tt + 1) / 2;
      for (int tile = tid; tile < ntiles; tile += NT) {
        int ti = static_cast<int>((sqrtf(8.0f * tile + 1.0f) - 1.0f) * 0.5f);
        while (ti * (ti + 1) / 2 > tile) --ti;
        while ((ti + 1) * (ti + 2) / 2 <= tile) ++ti;
        const int tj = tile - ti * (ti + 1) / 2;
        const int i0 = k1 + 4 * ti, j0 = k1 + 4 * tj;
        // rows past mr are clamped to mr - 1 and columns to the row (in-bounds loads, stores masked)
        int ri4[4], rj4[4], iq[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          iq[q] = min(i0 + q, mr - 1);
          ri4[q] = tri(iq[q]);
          rj4[q] = tri(min(j0 + q, mr - 1));
        }
        double acc[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int r = 0; r < 4; ++r) acc[q][r] = M[ri4[q] + min(j0 + r, iq[q])];
        for (int k = k0; k < k1; ++k) {
          const double inv = vinv[k];
          double li[4], lj[4];
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            li[q] = M[ri4[q] + k] * inv;
            lj[q] = M[rj4[q] + k];
          }
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int r = 0; r < 4; ++r) acc[q][r] -= li[q] * lj[r];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int r = 0; r < 4; ++r)
            if (i0 + q < mr && j0 + r <= i0 + q) M[ri4[q] + j0 + r] = acc[q][r];
      }
      __syncthreads();
    }
  };

  // ---- solve L D L' z = rhs in place (warp 0) ----
  // Lane l holds rows l, l + 32, l + 64, l + 96 of z (and of 1/D) in registers; step k broadcasts
  // the finished entry with a shuffle, so the serial chain per step is shuffle + FMA with the
  // shared-memory loads of L~ off the chain. Same operations, in the same order, as the
  // row-at-a-time substitution: forward w_k = z_k / D_k, z_i -= L~_ik w_k (L~ = L D); backward
  // x_k = w_k - (1/D_k) sum_{j>k} L~_jk x_j.
  // fwd_done: the forward substitution was done by an augmented factorization (row m of M holds
  // L^-1 rhs), so w = D^-1 (row m) and only the backward substitution runs.
  auto solve = [&](bool fwd_done) {
    if (warp == 0) {
      double zr[4], ir[4], ar[4];
      int ro[4];
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = t * 32 + lane;
        ir[t] = i < m ? vinv[i] : 0.0;
        zr[t] = i < m ? (fwd_done ? M[tri(m) + i] * ir[t] : vz[i]) : 0.0;
        ar[t] = 0.0;
        ro[t] = tri(min(i, m - 1));
      }
#pragma unroll
      for (int t = 0; t < 4 && !fwd_done; ++t) {
        const int kend = min(32, m - t * 32);
        for (int kk = 0; kk < kend; ++kk) {
          const int k = t * 32 + kk;
          const double wk = __shfl_sync(0xffffffffu, zr[t], kk) * __shfl_sync(0xffffffffu, ir[t], kk);
          if (lane == kk) zr[t] = wk;
#pragma unroll
          for (int u = t; u < 4; ++u) {
            const int i = u * 32 + lane;
            if (i > k && i < m) zr[u] -= M[ro[u] + k] * wk;
          }
        }
      }
#pragma unroll
      for (int t = 3; t >= 0; --t) {
        const int kstart = min(31, m - 1 - t * 32);
        for (int kk = kstart; kk >= 0; --kk) {
          const int k = t * 32 + kk;
          const double own = zr[t] - ir[t] * ar[t];
          const double xk = __shfl_sync(0xffffffffu, own, kk);
          if (lane == kk) zr[t] = xk;
          const int rk = tri(k);
#pragma unroll
          for (int u = 0; u <= t; ++u) {
            const int i = u * 32 + lane;
            if (i < k) ar[u] += M[rk + i] * xk;
          }
        }
      }
#pragma unroll
      for (int t = 0; t < 4; ++t) {
        const int i = t * 32 + lane;
        if (i < m) vz[i] = zr[t];
      }
    }
    __syncthreads();
  };

  // sum_p a_pj v[row_p] over column j from its record: the first two entries (missing ones as
  // 0 * v[0]) need no load that waits on another, the rest of a longer column follows from col_ptr
  auto col_dot = [&](const int4 rc, const double2 av, const double* v) {
    double acc = av.x * v[rc.x] + av.y * v[rc.y];
    for (int p = rc.z + 2; p < rc.w; ++p) acc += cv[p] * v[ri[p]];
    return acc;
  };
  constexpr int U = 3;  // columns per thread per pass, loads issued before use

  // ---- Mehrotra-like start (interior_point.cpp:488-506) ----
  // per-column scratch of an iteration: d = x/s in ds and t = d rd - rxs/s in dx for the
  // predictor's row pass, then w = 1/s in ds and t0 in dx for the corrector's (both free between
  // the update of one iteration and the corrector's direction pass that overwrites them)
  double* dvec = ds;
  double* tvec = dx;
  auto mehrotra_start = [&]() {
    for (int i = tid; i < tri(m + 1); i += NT) M[i] = 0.0;
    __syncthreads();
    for (int j = tid; j < n; j += NT) offdiag_rec(crc[j], cv2[j], 1.0);
    __syncthreads();
    row_pass(0, nullptr, nullptr);
    __syncthreads();
    factor(true);
    solve(true);
    const bool start_ok = !fail;
    for (int j = tid; j < n; j += NT) {
      double xs = 1.0, ss = 1.0;
      if (start_ok) {
        double atdy = 0.0;
        const int4 rc = crc[j];
        for (int p = rc.z; p < rc.w; ++p) atdy += cv[p] * vz[ri[p]];
        xs = fmax(1.0, fabs(atdy));
        ss = fmax(1.0, fabs(c[j] - atdy));
      }
      x[j] = xs;
      s[j] = ss;
      bx[j] = xs;
      bs[j] = ss;
    }
    for (int i = tid; i < m; i += NT) {
      vy[i] = start_ok ? vz[i] : 0.0;
      gby[i] = vy[i];
    }
    for (int i = tid; i < tri(m + 1); i += NT) M[i] = 0.0;
    fail = 0;
    __syncthreads();
  };
  for (int i = tid; i <= m; i += NT) srp[i] = rpp[i];  // visible after mehrotra_start's first barrier
  mehrotra_start();

  const int ops_res[4] = {1, 1, 0, 0};
  // ---- caller-supplied start (a learned prediction, a neighbouring LP's iterate) ----
  // Same rule as the single-problem engine: kept when its residual metric is within 10x of the
  // Mehrotra start's and its complementarity mu is not larger; otherwise the Mehrotra start stays.
  int warm_used = 0;
  if (mt.w_off >= 0) {
    // residual metric max(p_res, d_res, gap) and mu of the point in (x, vy, s)
    auto point_metric = [&](double& metric, double& mu) {
      double rpm = 0.0;
      for (int i = warp; i < m; i += NW) {
        double acc = 0.0;
        for (int p = srp[i] + lane; p < srp[i + 1]; p += 32) acc += rv[p] * x[ci[p]];
        acc = warp_sum(acc);
        rpm = fmax(rpm, fabs(b[i] - acc));
      }
      double rdm = 0.0, xs = 0.0, cx = 0.0;
      for (int j = tid; j < n; j += NT) {
        const double r = c[j] - (col_dot(crc[j], cv2[j], vy) + s[j]);
        rdm = fmax(rdm, fabs(r));
        xs += x[j] * s[j];
        cx += c[j] * x[j];
      }
      double v[4] = {rpm, rdm, xs, cx};
      cta_reduce4<NT>(v, ops_res, red);
      if (tid == 0) {
        cs.v[S_MU] = v[2] / n;
        cs.v[S_METRIC] = fmax(fmax(v[0] / mt.bnorm, v[1] / mt.cnorm), fabs(v[2]) / (1.0 + fabs(v[3])));
      }
      __syncthreads();
      metric = cs.v[S_METRIC];
      mu = cs.v[S_MU];
      __syncthreads();
    };
    double met_d, mu_d, met_w, mu_w;
    point_metric(met_d, mu_d);
    const double* wx = bd.warm + mt.w_off;
    for (int j = tid; j < n; j += NT) {
      x[j] = wx[j];
      s[j] = wx[n + m + j];
    }
    for (int i = tid; i < m; i += NT) vy[i] = wx[n + i];
    __syncthreads();
    point_metric(met_w, mu_w);
    if (isfinite(met_w) && isfinite(mu_w) && met_w <= 10.0 * met_d && mu_w <= mu_d) {
      warm_used = 1;
    } else {
      for (int j = tid; j < n; j += NT) {
        x[j] = bx[j];
        s[j] = bs[j];
      }
      for (int i = tid; i < m; i += NT) vy[i] = gby[i];
    }
    __syncthreads();
  }

  double best_metric = INFINITY, best_gap = INFINITY, best_p = INFINITY, best_d = INFINITY;
  int best_it = 0;
  int status = -1, iters = 0;
  double last_gap = 0, last_p = 0, last_d = 0, last_cx = 0;
  for (int it = 0; it < mt.max_iter; ++it) {
    // residuals, with the predictor's right-hand side and the normal matrix built in the same two
    // passes (interior_point.cpp:572-582, :418-432, :74-101)
    double rdm = 0.0, xs = 0.0, cx = 0.0;
    for (int j0 = tid; j0 < n; j0 += U * NT) {
      int4 rc[U];
      double2 av[U];
      double xv[U], sv[U], cvv[U], aty[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = min(j0 + u * NT, n - 1);
        rc[u] = crc[j];
        av[u] = cv2[j];
        xv[u] = x[j];
        sv[u] = s[j];
        cvv[u] = c[j];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) aty[u] = col_dot(rc[u], av[u], vy);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = j0 + u * NT;
        if (j >= n) continue;
        const double r = cvv[u] - (aty[u] + sv[u]);
        rd[j] = r;
        rdm = fmax(rdm, fabs(r));
        xs += xv[u] * sv[u];
        cx += cvv[u] * xv[u];
        const double xj = fmax(xv[u], 1e-16), sj = fmax(sv[u], 1e-16);
        const double dj = xj / sj;
        const double rxs = -xv[u] * sv[u];
        dvec[j] = dj;
        tvec[j] = dj * r - rxs / sj;
        offdiag_rec(rc[u], av[u], dj);
      }
    }
    __syncthreads();
    const double rpm = row_pass(1, dvec, tvec);
    double v[4] = {rpm, rdm, xs, cx};
    cta_reduce4<NT>(v, ops_res, red);
    if (tid == 0) {
      const double mu = v[2] / n;
      const double pres = v[0] / mt.bnorm, dres = v[1] / mt.cnorm;
      const double gap = fabs(v[2]) / (1.0 + fabs(v[3]));
      cs.v[S_MU] = mu;
      cs.v[S_PRES] = pres;
      cs.v[S_DRES] = dres;
      cs.v[S_GAP] = gap;
      cs.v[S_METRIC] = fmax(pres, fmax(dres, gap));
      cs.v[S_CX] = v[3];
    }
    __syncthreads();
    const double mu = cs.v[S_MU], pres = cs.v[S_PRES], dres = cs.v[S_DRES], gap = cs.v[S_GAP];
    const double metric = cs.v[S_METRIC];
    last_gap = gap;
    last_p = pres;
    last_d = dres;
    last_cx = cs.v[S_CX];
    if (metric < best_metric) {
      best_metric = metric;
      best_gap = gap;
      best_p = pres;
      best_d = dres;
      best_it = it + 1;
      for (int j = tid; j < n; j += NT) {
        bx[j] = x[j];
        bs[j] = s[j];
      }
      for (int i = tid; i < m; i += NT) gby[i] = vy[i];
    }
    if (gap < best_gap) best_gap = gap;
    if (pres < mt.ftol && dres < mt.ftol && gap < mt.otol) {
      status = SOV_OPTIMAL;
      iters = it + 1;
      break;
    }
    // a supplied start that has not converged after kWarmGiveUp iterations is abandoned once: the
    // LP restarts from the Mehrotra start (its best-iterate record restarts too), so one poor
    // prediction costs at most kWarmGiveUp extra iterations instead of running to the limit
    if (warm_used == 1 && it + 1 == kWarmGiveUp) {
      mehrotra_start();
      warm_used = 2;
      best_metric = best_gap = best_p = best_d = INFINITY;
      best_it = 0;
      continue;
    }
    // factor A diag(x/s) A' (assembled by the residual passes), with the predictor's right-hand
    // side as the augmented row
    factor(true);
    if (fail) {
      status = -2;  // factorization failure: best iterate
      break;
    }
    // predictor and corrector
    //  predictor: solve, then one column pass for the affine direction, its step-length ratios and
    //    the four sums that give mu_aff = (1/n) sum (x + a_p dx)(s + a_d ds) once the steps are
    //    known (sum xs + a_p sum dx s + a_d sum x ds + a_p a_d sum dx ds); the same pass leaves the
    //    corrector's right-hand side as t0 = d rd + (x s + dx_aff ds_aff)/s and w = 1/s, so that
    //    t = d rd - rxs/s with rxs = -x s - dx_aff ds_aff + sigma mu (interior_point.cpp:676-681)
    //    is t0 - sigma mu w, formed inside the row pass z = rp + A t;
    //  corrector: that row pass, solve, one column pass for the direction and the step lengths.
    for (int pass = 0; pass < 2; ++pass) {
      const double sigma_mu = pass ? cs.v[S_SIGMA] * mu : 0.0;
      if (pass == 1) {
        row_pass(2, dvec, tvec, sigma_mu);
        __syncthreads();
      }
      solve(pass == 0);
      double* ddx = pass ? dx : dxa;
      double* dds = pass ? ds : dsa;
      double rpmin = 1.0, rdmin = 1.0, sxs = 0.0, sdxs = 0.0, sxds = 0.0, sdd = 0.0;
      for (int j0 = tid; j0 < n; j0 += U * NT) {
        int4 rc[U];
        double2 cav[U];
        double xv[U], sv[U], rdv[U], av[U], bv[U], atdy[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = min(j0 + u * NT, n - 1);
          rc[u] = crc[j];
          cav[u] = cv2[j];
          xv[u] = x[j];
          sv[u] = s[j];
          rdv[u] = rd[j];
          av[u] = pass ? dxa[j] : 0.0;
          bv[u] = pass ? dsa[j] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) atdy[u] = col_dot(rc[u], cav[u], vz);
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int j = j0 + u * NT;
          if (j >= n) continue;
          const double xj = xv[u], sj = sv[u];
          const double rxs = pass ? -xj * sj - av[u] * bv[u] + sigma_mu : -xj * sj;
          const double sg = fmax(sj, 1e-16);
          const double dj = fmax(xj, 1e-16) / sg;
          const double dxj = dj * (atdy[u] - rdv[u]) + rxs / sg;
          const double dsj = rdv[u] - atdy[u];
          ddx[j] = dxj;
          dds[j] = dsj;
          if (dxj < 0.0) rpmin = fmin(rpmin, -xj / dxj);
          if (dsj < 0.0) rdmin = fmin(rdmin, -sj / dsj);
          if (pass == 0) {
            sxs += xj * sj;
            sdxs += dxj * sj;
            sxds += xj * dsj;
            sdd += dxj * dsj;
            tvec[j] = dj * rdv[u] + (xj * sj + dxj * dsj) / sg;
            dvec[j] = 1.0 / sg;
          }
        }
      }
      if (pass == 0) {
        double u[6] = {rpmin, rdmin, sxs, sdxs, sxds, sdd};
        const int ops[6] = {2, 2, 0, 0, 0, 0};
        block_reduce<6>(u, ops, red);
        if (tid == 0) {
          const double apa = u[0], ada = u[1];
          cs.v[S_APAFF] = apa;
          cs.v[S_ADAFF] = ada;
          const double mu_aff = fmax(0.0, u[2] + apa * u[3] + ada * u[4] + apa * ada * u[5]) / n;
          const double r = mu_aff / mu;
          cs.v[S_SIGMA] = mu > 0.0 ? fmin(1.0, r * r * r) : 0.0;
        }
      } else {
        double u[4] = {rpmin, rdmin, 0.0, 0.0};
        const int ops_min[4] = {2, 2, 0, 0};
        cta_reduce4<NT>(u, ops_min, red);
        if (tid == 0) {
          cs.v[S_AP] = fmin(1.0, mt.tau * u[0]);
          cs.v[S_AD] = fmin(1.0, mt.tau * u[1]);
        }
      }
      __syncthreads();
    }
    // update (interior_point.cpp:709-718)
    const double ap = cs.v[S_AP], ad = cs.v[S_AD];
    for (int j0 = tid; j0 < n; j0 += U * NT) {
      double xv[U], sv[U], av[U], bv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = min(j0 + u * NT, n - 1);
        xv[u] = x[j];
        sv[u] = s[j];
        av[u] = dx[j];
        bv[u] = ds[j];
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int j = j0 + u * NT;
        if (j >= n) continue;
        x[j] = fmax(xv[u] + ap * av[u], 1e-14);
        s[j] = fmax(sv[u] + ad * bv[u], 1e-14);
      }
    }
    for (int i = tid; i < m; i += NT) vy[i] += ad * vz[i];
    for (int i = tid; i < tri(m + 1); i += NT) M[i] = 0.0;
    iters = it + 1;
    __syncthreads();
  }
  for (int i = tid; i < m; i += NT) gy[i] = vy[i];
  if (tid == 0) {
    LpOut o{};
    o.drops = drops;
    o.fail = fail;
    o.warm_used = warm_used == 1 ? 1 : 0;
    if (status == SOV_OPTIMAL) {
      o.status = SOV_OPTIMAL;
      o.iterations = iters;
      o.use_best = 0;
      o.gap = last_gap;
      o.p_res = last_p;
      o.d_res = last_d;
    } else {
      o.status = best_p <= mt.ftol ? SOV_FEASIBLE : SOV_NUMERICAL_ERROR;
      o.iterations = best_it;
      o.use_best = 1;
      o.best_it = status == -2 ? 1 : 0;  // 1: stopped on a failed factorization
      o.gap = best_gap;
      o.p_res = best_p;
      o.d_res = best_d;
    }
    o.cx = last_cx;
    bd.out[lp] = o;
  }
  __syncthreads();
}

// Kernel shapes: the CTA width NT and the CTAs per SM its register budget is sized for. The plain
// shapes get 128 registers per thread (4 x 128, 2 x 256, 1 x 512 threads per SM); the lean ones
// are capped at 80 registers (6 x 128, 3 x 256 per SM), which spills a little but keeps more LPs
// resident to cover each other's barrier waits. A shape code is the width, plus 1 for lean.
constexpr int min_ctas(int nt, bool lean) { return lean ? (nt <= 128 ? 6 : 3) : (nt <= 128 ? 4 : nt <= 256 ? 2 : 1); }
constexpr int kShapes[] = {128, 129, 256, 257, 512};

template <int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) k_batch_ipm(BatchDev bd, int mmax) {
  extern __shared__ double sm[];
  __shared__ double red[6 * 32];
  __shared__ CtaScalars cs;
  __shared__ int slot_s;
  for (;;) {
    if (threadIdx.x == 0) slot_s = atomicAdd(bd.next, 1);
    __syncthreads();
    const int slot = slot_s;
    __syncthreads();
    if (slot >= bd.count) return;
    const int lp = bd.order[slot];
    solve_lp<NT>(bd, bd.meta[lp], lp, sm, mmax, red, cs);
  }
}

// packed triangle (with the augmented row) | six m-vectors | m + 1 row pointers
size_t batch_smem(int mmax) {
  return sizeof(double) * (static_cast<size_t>(tri(mmax + 1)) + 6 * mmax) + sizeof(int) * (mmax + 2);
}

// The dynamic shared-memory limit of every instantiation is raised once to the largest bucket's
// footprint, so launches (and launches captured in a graph) need no per-launch attribute call.
void ensure_smem_limits() {
  const int smem = static_cast<int>(batch_smem(kBatchMaxRows));
  once_per_device((const void*)k_batch_ipm<128, min_ctas(128, false)>, [&] {
    SOV_CUDA(cudaFuncSetAttribute(k_batch_ipm<128, min_ctas(128, false)>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    SOV_CUDA(cudaFuncSetAttribute(k_batch_ipm<128, min_ctas(128, true)>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    SOV_CUDA(cudaFuncSetAttribute(k_batch_ipm<256, min_ctas(256, false)>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    SOV_CUDA(cudaFuncSetAttribute(k_batch_ipm<256, min_ctas(256, true)>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    SOV_CUDA(cudaFuncSetAttribute(k_batch_ipm<512, min_ctas(512, false)>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  });
}

template <int NT, bool LEAN>
void launch_bucket(const BatchDev& bd, int mmax, int grid, cudaStream_t st) {
  k_batch_ipm<NT, min_ctas(NT, LEAN)><<<grid, NT, batch_smem(mmax), st>>>(bd, mmax);
  SOV_LAUNCH_CHECK();
}

template <int NT, bool LEAN>
int max_ctas(int mmax) {
  int per_sm = 0;
  const size_t smem = batch_smem(mmax);
  SOV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_ipm<NT, min_ctas(NT, LEAN)>, NT, smem));
  int dev = 0, sms = 0;
  SOV_CUDA(cudaGetDevice(&dev));
  SOV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return std::max(1, per_sm) * sms;
}

// Per-device cache of released device blocks: a batch created per end-to-end call (hundreds of MB
// of inputs and work vectors) reuses the previous call's memory instead of paying cudaMalloc and
// cudaFree each time. A block is reused for a request of at least half its size; at most
// kMaxCached bytes stay cached, and a failed cudaMalloc first returns the cache to the device.
// Blocks return to the cache only after the batch's work has finished (every batch operation is
// synchronous with respect to its own device memory).
class DevicePool {
 public:
  void* acquire(size_t bytes, size_t* got) {
    int dev = 0;
    SOV_CUDA(cudaGetDevice(&dev));
    {
      std::lock_guard<std::mutex> g(mu_);
      for (auto it = free_.lower_bound(bytes); it != free_.end() && it->first <= 2 * bytes + (1u << 20); ++it) {
        if (it->second.first != dev) continue;
        void* p = it->second.second;
        *got = it->first;
        cached_ -= it->first;
        free_.erase(it);
        return p;
      }
    }
    void* p = nullptr;
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      trim(0);
      SOV_CUDA(cudaMalloc(&p, bytes));
    }
    *got = bytes;
    return p;
  }
  void release(void* p, size_t bytes) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    {
      std::lock_guard<std::mutex> g(mu_);
      free_.emplace(bytes, std::make_pair(dev, p));
      cached_ += bytes;
    }
    trim(kMaxCached);
  }
  // free cached blocks (largest first) until at most `keep` bytes stay cached
  void trim(size_t keep) {
    std::lock_guard<std::mutex> g(mu_);
    while (cached_ > keep && !free_.empty()) {
      auto it = std::prev(free_.end());
      int cur = 0;
      cudaGetDevice(&cur);
      cudaSetDevice(it->second.first);
      cudaFree(it->second.second);
      cudaSetDevice(cur);
      cached_ -= it->first;
      free_.erase(it);
    }
  }

 private:
  static constexpr size_t kMaxCached = size_t(4) << 30;
  std::mutex mu_;
  std::multimap<size_t, std::pair<int, void*>> free_;
  size_t cached_ = 0;
};
DevicePool g_dpool;

template <class T>
struct DBuf {
  T* p = nullptr;
  size_t n = 0, cap_bytes = 0;
  void alloc(size_t count) {
    if (count) p = static_cast<T*>(g_dpool.acquire(sizeof(T) * count, &cap_bytes));
    n = count;
  }
  ~DBuf() {
    if (p) g_dpool.release(p, cap_bytes);
  }
};

// Host counterpart for per-batch host arrays (the publishing data of every LP): released blocks
// stay mapped and are reused, so building a batch does not page-fault fresh memory each call.
class HostPool {
 public:
  void* acquire(size_t bytes, size_t* got) {
    {
      std::lock_guard<std::mutex> g(mu_);
      auto it = free_.lower_bound(bytes);
      if (it != free_.end() && it->first <= 2 * bytes + (1u << 20)) {
        void* p = it->second;
        *got = it->first;
        cached_ -= it->first;
        free_.erase(it);
        return p;
      }
    }
    void* p = std::malloc(bytes);
    if (!p) throw std::bad_alloc();
    *got = bytes;
    return p;
  }
  void release(void* p, size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    free_.emplace(bytes, p);
    cached_ += bytes;
    while (cached_ > kMaxCached && !free_.empty()) {
      auto it = std::prev(free_.end());
      std::free(it->second);
      cached_ -= it->first;
      free_.erase(it);
    }
  }

 private:
  static constexpr size_t kMaxCached = size_t(2) << 30;
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  size_t cached_ = 0;
};
HostPool g_hpool;

template <class T>
struct HBuf {
  T* p = nullptr;
  size_t cap_bytes = 0;
  void alloc(size_t count) {
    if (count) p = static_cast<T*>(g_hpool.acquire(sizeof(T) * count, &cap_bytes));
  }
  ~HBuf() {
    if (p) g_hpool.release(p, cap_bytes);
  }
};

// Pinned host blocks for per-batch results (the statuses and published values of every LP, copied
// behind the publish kernel on the solve's stream): released blocks stay pinned and are reused, so
// a call pins no memory after the first few.
class PinnedPool {
 public:
  void* acquire(size_t bytes, size_t* got) {
    {
      std::lock_guard<std::mutex> g(mu_);
      auto it = free_.lower_bound(bytes);
      if (it != free_.end() && it->first <= 2 * bytes + (1u << 20)) {
        void* p = it->second;
        *got = it->first;
        cached_ -= it->first;
        free_.erase(it);
        return p;
      }
    }
    void* p = nullptr;
    SOV_CUDA(cudaMallocHost(&p, bytes));
    *got = bytes;
    return p;
  }
  void release(void* p, size_t bytes) {
    std::lock_guard<std::mutex> g(mu_);
    free_.emplace(bytes, p);
    cached_ += bytes;
    while (cached_ > kMaxCached && !free_.empty()) {
      auto it = std::prev(free_.end());
      cudaFreeHost(it->second);
      cached_ -= it->first;
      free_.erase(it);
    }
  }

 private:
  static constexpr size_t kMaxCached = size_t(1) << 30;
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  size_t cached_ = 0;
};
PinnedPool g_ppool;

template <class T>
struct PBuf {
  T* p = nullptr;
  size_t cap_bytes = 0;
  void alloc(size_t count) {
    if (count && !p) p = static_cast<T*>(g_ppool.acquire(sizeof(T) * count, &cap_bytes));
  }
  ~PBuf() {
    if (p) g_ppool.release(p, cap_bytes);
  }
};

// Grow-only pinned host stagings shared by all batches of the process (H2D of the packed inputs,
// D2H of the iterates), so repeated end-to-end calls do not re-pin memory. Two of them, taken in
// turn: a batch leaves its input copies in flight (`pending`) and the next batch builds into the
// other staging, so the building of one part of a pipelined call overlaps the copies of the one
// before. Whoever takes a staging next waits for its pending copies first.
struct PinnedArena {
  std::mutex mu;
  unsigned char* p = nullptr;
  size_t cap = 0;
  cudaEvent_t pending = nullptr;  // recorded behind the last async copies out of `p`
  int pending_dev = -1;
  unsigned char* get(size_t bytes) {
    if (pending) SOV_CUDA(cudaEventSynchronize(pending));
    if (bytes > cap) {
      if (p) cudaFreeHost(p);
      p = nullptr;
      cap = 0;
      SOV_CUDA(cudaMallocHost(&p, bytes));
      cap = bytes;
    }
    return p;
  }
  // mark the copies enqueued on `st` so far as readers of the staging
  void record(cudaStream_t st) {
    int dev = 0;
    SOV_CUDA(cudaGetDevice(&dev));
    if (pending && pending_dev != dev) {
      cudaEventDestroy(pending);
      pending = nullptr;
    }
    if (!pending) {
      SOV_CUDA(cudaEventCreateWithFlags(&pending, cudaEventDisableTiming));
      pending_dev = dev;
    }
    SOV_CUDA(cudaEventRecord(pending, st));
  }
};
PinnedArena g_arenas[2];
std::atomic<unsigned> g_arena_turn{0};

std::mutex g_tune_mu;
std::map<int, int> g_tuned_threads;  // bucket mmax -> kernel shape code
std::map<int, int> g_tuned_per_sm;   // bucket mmax -> resident CTAs per SM it launches (absent: all that fit)

int bucket_of(int m) { return std::max(32, ((m + 31) / 32) * 32); }

// Host worker threads, started once and kept for the life of the process (never destroyed: they
// wait on a condition variable when idle): the batch builds and publishes run several parallel
// loops per call, and starting threads for each of them cost milliseconds per call. One loop at a
// time uses the pool; a loop that finds it busy (another host thread's batch), or runs in a forked
// child (which has none of the parent's threads), runs on its own thread instead.
class WorkerPool {
 public:
  static WorkerPool& get() {
    static WorkerPool* pool = new WorkerPool;
    return *pool;
  }
  int width() const { return static_cast<int>(threads_.size()) + 1; }
  // fn(i) for i in [0, count) on the workers and the calling thread; false when the pool is busy
  bool run(int count, const std::function<void(int)>& fn) {
    if (getpid() != owner_) return false;
    std::unique_lock<std::mutex> job(busy_, std::try_to_lock);
    if (!job.owns_lock()) return false;
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      count_ = count;
      next_.store(0);
      error_.clear();
      active_ = static_cast<int>(threads_.size());
      ++generation_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [&] { return active_ == 0; });
    fn_ = nullptr;
    if (!error_.empty()) throw std::runtime_error(error_);
    return true;
  }

 private:
  WorkerPool() : owner_(getpid()) {
    const int nt = std::max(1, std::min<int>(16, static_cast<int>(std::thread::hardware_concurrency())));
    for (int w = 1; w < nt; ++w) threads_.emplace_back([this] { loop(); });
  }
  void work() {
    for (int i = next_.fetch_add(1); i < count_; i = next_.fetch_add(1)) {
      try {
        (*fn_)(i);
      } catch (const std::exception& e) {
        std::lock_guard<std::mutex> lk(err_mu_);
        if (error_.empty()) error_ = e.what();
        next_.store(count_);
      }
    }
  }
  void loop() {
    unsigned long long seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return generation_ != seen; });
        seen = generation_;
      }
      work();
      std::lock_guard<std::mutex> lk(mu_);
      if (--active_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> threads_;
  std::mutex busy_, mu_, err_mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)>* fn_ = nullptr;
  int count_ = 0, active_ = 0;
  std::atomic<int> next_{0};
  unsigned long long generation_ = 0;
  std::string error_;
  const pid_t owner_;
};

// the device's highest stream priority (numerically the least value)
int high_priority() {
  int least = 0, greatest = 0;
  SOV_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  return greatest;
}

// Streams and events made once per process and reused: a call solved in six parts made and
// destroyed about 80 of them, 1.9 ms of a 23 ms call. An object goes back only when the work
// queued on it has completed (its batch finished and read back, or synchronized after an error).
class CudaObjectPool {
 public:
  static CudaObjectPool& get() {
    static CudaObjectPool* pool = new CudaObjectPool;  // never destroyed: no CUDA calls at exit
    return *pool;
  }
  cudaStream_t stream(bool high) {
    {
      std::lock_guard<std::mutex> g(mu_);
      auto& v = high ? high_ : normal_;
      if (!v.empty()) {
        cudaStream_t st = v.back();
        v.pop_back();
        return st;
      }
    }
    cudaStream_t st = nullptr;
    if (high) SOV_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, high_priority()));
    else SOV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    return st;
  }
  cudaEvent_t event(bool timing) {
    {
      std::lock_guard<std::mutex> g(mu_);
      auto& v = timing ? timed_ : untimed_;
      if (!v.empty()) {
        cudaEvent_t e = v.back();
        v.pop_back();
        return e;
      }
    }
    cudaEvent_t e = nullptr;
    SOV_CUDA(cudaEventCreateWithFlags(&e, timing ? cudaEventDefault : cudaEventDisableTiming));
    return e;
  }
  void give_stream(cudaStream_t st, bool high) {
    if (!st) return;
    std::lock_guard<std::mutex> g(mu_);
    (high ? high_ : normal_).push_back(st);
  }
  void give_event(cudaEvent_t e, bool timing) {
    if (!e) return;
    std::lock_guard<std::mutex> g(mu_);
    (timing ? timed_ : untimed_).push_back(e);
  }

 private:
  std::mutex mu_;
  std::vector<cudaStream_t> normal_, high_;
  std::vector<cudaEvent_t> timed_, untimed_;
};

template <class F>
void parallel_for(int count, F fn) {
  if (count < 64) {
    for (int i = 0; i < count; ++i) fn(i);
    return;
  }
  const std::function<void(int)> f = fn;
  if (WorkerPool::get().width() > 1 && WorkerPool::get().run(count, f)) return;
  for (int i = 0; i < count; ++i) fn(i);
}

}  // namespace

struct Batch {
  int count = 0;
  std::vector<sov_model> models;
  std::vector<StdForm> forms;  // only for LPs not built in place (non-plain columns, or too large)
  std::vector<LpMeta> meta;
  // publishing (interior_point.cpp:521-569): per LP its sizes and where its shift sits in
  // `pubdata` (followed by room for the unit scales the in-place builder writes; the scales used
  // are on the device, `scl`)
  struct Pub {
    int n_struct, m0, n, m;
    long long shift_off, cs_off, rs_off;
    LpFormInfo info;
  };
  std::vector<Pub> pub;
  HBuf<double> pubdata;
  std::vector<int> fallback;  // LPs too large for the batched kernel
  // starts handed over on the device (DeviceStarts), kept for the fallback LPs, which take theirs
  // as host warm starts
  bool has_dstarts = false;
  DeviceStarts dstarts{};
  int first_lp = 0;
  sov_options opt{};
  std::vector<sov_options> opts;  // per-LP options (empty: `opt` for all)
  struct Bucket {
    int mmax, threads, grid, count;
    const int* order;  // device: this bucket's LP indices, largest first (inside `in`)
    int* next;         // device: its work counter (inside `nexts`)
  };
  std::vector<std::unique_ptr<Bucket>> buckets;
  // one device arena for all packed inputs: [meta | ints | doubles | bucket orders]
  DBuf<unsigned char> in;
  DBuf<double> work;  // 9 n-vectors + 2 m-vectors
  DBuf<int4> crec;     // column records (BatchDev::crec), built by k_batch_rows
  DBuf<double2> cval2;
  DBuf<LpOut> out;
  DBuf<int> nexts;
  // published scale products of every LP (k_batch_publish), then per LP the coefficient range
  // after scaling (k_batch_scale)
  DBuf<double> pout;
  // host copies of `out` and `pout`, made on the solve's stream behind k_batch_publish (the
  // `published` event covers them), so reading results waits for no copy of its own
  PBuf<LpOut> h_out;
  PBuf<double> h_pout;
  double* scl = nullptr;  // device: column scales (total_n) | row scales (total_m), inside `in`
  long long total_n = 0, total_m = 0, total_nnz = 0, total_cols = 0, total_rows = 0, total_pub = 0;
  BatchDev dev{};
  int launches = 0;
  double kernel_ms = 0.0, bytes = 0.0, flops = 0.0;
  double h2d_bytes = 0.0, d2h_bytes = 0.0;
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
  cudaEvent_t ready = nullptr;      // inputs scaled and row copies built (k_batch_scale, k_batch_rows)
  cudaEvent_t published = nullptr;  // k_batch_publish of the last solve done
  bool publish_queued = false;      // k_batch_publish already enqueued behind the last solve
  cudaStream_t input_stream = nullptr;  // the input copies and kernels (high priority)
  cudaStream_t cap = nullptr;
  cudaGraphExec_t graph = nullptr;  // the bucket launches of one solve
  ~Batch() {
    if (graph) cudaGraphExecDestroy(graph);
    // the input kernels write the device buffers released below (a batch destroyed unsolved)
    if (ready) cudaEventSynchronize(ready);
    // the result copies into h_out / h_pout (released below) follow the publish kernel
    if (published) cudaEventSynchronize(published);
    if (cap) cudaStreamDestroy(cap);
    CudaObjectPool& pool = CudaObjectPool::get();
    for (auto st : streams) pool.give_stream(st, false);
    for (auto e : joins) pool.give_event(e, false);
    pool.give_event(fork, false);
    pool.give_event(t0, true);
    pool.give_event(t1, true);
    pool.give_event(ready, false);
    pool.give_event(published, false);
    pool.give_stream(input_stream, true);
  }
};

namespace {

// The row-wise copy (col_idx, rval) of every batched LP from its columns, and the column records
// (BatchDev::crec, cval2), one CTA per LP, on the
// device: the host sends the columns and the row starts only. Columns are taken in chunks of
// 256 in ascending order; in a chunk, thread t (column c0 + t) sets bit t of each of its rows'
// masks, and an entry's place in its row is the row's running count plus the bits below t, so
// every row lists its columns in ascending order, exactly as the host's fill does.
constexpr int kRowsThreads = 256;

__global__ void __launch_bounds__(kRowsThreads) k_batch_rows(const LpMeta* __restrict__ meta, const int* __restrict__ cpa,
                                                             const int* __restrict__ ria, const double* __restrict__ cva,
                                                             const int* __restrict__ rpa, int* __restrict__ cia,
                                                             double* __restrict__ rva, int4* __restrict__ crec,
                                                             double2* __restrict__ cval2) {
  __shared__ unsigned mask[kBatchMaxRows][kRowsThreads / 32];
  __shared__ int base[kBatchMaxRows];
  const LpMeta mt = meta[blockIdx.x];
  if (mt.m < 0) return;
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
  const int* cp = cpa + mt.cp_off;
  const int* ri = ria + mt.a_off;
  const double* cv = cva + mt.a_off;
  const int* rp = rpa + mt.rp_off;
  int* ci = cia + mt.a_off;
  double* rv = rva + mt.a_off;
  for (int r = tid; r < mt.m; r += kRowsThreads) base[r] = rp[r];
  for (int c0 = 0; c0 < mt.n; c0 += kRowsThreads) {
    for (int q = tid; q < mt.m * (kRowsThreads / 32); q += kRowsThreads) mask[q / (kRowsThreads / 32)][q % (kRowsThreads / 32)] = 0u;
    __syncthreads();
    const int j = c0 + tid;
    const int pb = j < mt.n ? cp[j] : 0, pe = j < mt.n ? cp[j + 1] : 0;
    if (j < mt.n) {
      const bool h0 = pb < pe, h1 = pb + 1 < pe;
      crec[mt.nv_off + j] = make_int4(h0 ? ri[pb] : 0, h1 ? ri[pb + 1] : 0, pb, pe);
      cval2[mt.nv_off + j] = make_double2(h0 ? cv[pb] : 0.0, h1 ? cv[pb + 1] : 0.0);
    }
    for (int p = pb; p < pe; ++p) atomicOr(&mask[ri[p]][w], 1u << lane);
    __syncthreads();
    for (int p = pb; p < pe; ++p) {
      const int r = ri[p];
      int rank = __popc(mask[r][w] & ((1u << lane) - 1u));
      for (int v = 0; v < w; ++v) rank += __popc(mask[r][v]);
      const int at = base[r] + rank;
      ci[at] = j;
      rv[at] = cv[p];
    }
    __syncthreads();
    for (int r = tid; r < mt.m; r += kRowsThreads) {
      int c = 0;
#pragma unroll
      for (int v = 0; v < kRowsThreads / 32; ++v) c += __popc(mask[r][v]);
      base[r] += c;
    }
    __syncthreads();
  }
}

// The two-pass scaling of every batched LP built in place (interior_point.cpp:370-405: rows by
// 1/sqrt(max|a|), then columns, twice), one CTA per LP, on the device: the host sends the unscaled
// columns. Every value sees the host builder's products in the host builder's order, and the row,
// column and range maxima are exact whatever order the threads take (a NaN never replaces a running
// maximum, as in std::max(cur, a)), so values, b, c, the scales and the coefficient range are bit
// for bit the host's. Also, for every LP, bnorm = max(1, max|b|) and cnorm = max(1, max|c|) of the
// scaled data (interior_point.cpp:586).
constexpr int kScaleThreads = 256;

__device__ __forceinline__ double inv_sqrt_or_one(double x) { return x > 0.0 ? 1.0 / sqrt(x) : 1.0; }

// running maximum of non-negative doubles held as their bit patterns (ordered like the values)
__device__ __forceinline__ void max_bits(unsigned long long* slot, double a) {
  if (a > 0.0) atomicMax(slot, static_cast<unsigned long long>(__double_as_longlong(a)));
}

__global__ void __launch_bounds__(kScaleThreads) k_batch_scale(LpMeta* __restrict__ meta, const int* __restrict__ cpa,
                                                               const int* __restrict__ ria, double* __restrict__ cva,
                                                               double* __restrict__ ba, double* __restrict__ ca,
                                                               double* __restrict__ scl, long long total_n,
                                                               double* __restrict__ crange) {
  __shared__ unsigned long long rmax[kBatchMaxRows];
  __shared__ double rsc[kBatchMaxRows];
  __shared__ unsigned long long lo_bits, hi_bits, bmax_bits, cmax_bits;
  LpMeta* mp = meta + blockIdx.x;
  const int m = mp->m, n = mp->n, mode = mp->scale_mode;
  if (m < 0) return;
  const int tid = threadIdx.x;
  const int* cp = cpa + mp->cp_off;
  const int* ri = ria + mp->a_off;
  double* cv = cva + mp->a_off;
  double* b = ba + mp->mv_off;
  double* c = ca + mp->nv_off;
  double* cs = scl + mp->nv_off;
  double* rs = scl + total_n + mp->mv_off;
  constexpr unsigned long long inf_bits = 0x7ff0000000000000ull;  // +infinity
  if (tid == 0) {
    lo_bits = inf_bits;
    hi_bits = 0ull;
    bmax_bits = 0ull;
    cmax_bits = 0ull;
  }
  if (mode == 1) {
    for (int r = tid; r < m; r += kScaleThreads) rmax[r] = 0ull;
    __syncthreads();
    for (int j = tid; j < n; j += kScaleThreads)
      for (int p = cp[j]; p < cp[j + 1]; ++p) max_bits(&rmax[ri[p]], fabs(cv[p]));
    for (int pass = 0; pass < 2; ++pass) {
      __syncthreads();
      for (int r = tid; r < m; r += kScaleThreads) {
        const double f = inv_sqrt_or_one(__longlong_as_double(static_cast<long long>(rmax[r])));
        rsc[r] = f;
        rs[r] = pass == 0 ? f : __dmul_rn(rs[r], f);
        b[r] = __dmul_rn(b[r], f);
        rmax[r] = 0ull;
      }
      __syncthreads();
      for (int j = tid; j < n; j += kScaleThreads) {
        const int pb = cp[j], pe = cp[j + 1];
        double mx = 0.0;
        for (int p = pb; p < pe; ++p) {
          const double v = __dmul_rn(cv[p], rsc[ri[p]]);
          cv[p] = v;
          const double a = fabs(v);
          mx = mx < a ? a : mx;
        }
        const double f = inv_sqrt_or_one(mx);
        for (int p = pb; p < pe; ++p) {
          const double v = __dmul_rn(cv[p], f);
          cv[p] = v;
          const double a = fabs(v);
          if (pass == 0) {
            max_bits(&rmax[ri[p]], a);
          } else if (a > 0.0 && a <= DBL_MAX) {
            const unsigned long long ab = static_cast<unsigned long long>(__double_as_longlong(a));
            atomicMin(&lo_bits, ab);
            atomicMax(&hi_bits, ab);
          }
        }
        c[j] = __dmul_rn(c[j], f);
        cs[j] = pass == 0 ? f : __dmul_rn(cs[j], f);
      }
    }
  } else if (mode == 0) {
    for (int j = tid; j < n; j += kScaleThreads) cs[j] = 1.0;
    for (int r = tid; r < m; r += kScaleThreads) rs[r] = 1.0;
  }
  __syncthreads();
  for (int r = tid; r < m; r += kScaleThreads) max_bits(&bmax_bits, fabs(b[r]));
  for (int j = tid; j < n; j += kScaleThreads) max_bits(&cmax_bits, fabs(c[j]));
  __syncthreads();
  if (tid == 0) {
    const double bm = __longlong_as_double(static_cast<long long>(bmax_bits));
    const double cm = __longlong_as_double(static_cast<long long>(cmax_bits));
    mp->bnorm = 1.0 < bm ? bm : 1.0;
    mp->cnorm = 1.0 < cm ? cm : 1.0;
    crange[2 * blockIdx.x] = __longlong_as_double(static_cast<long long>(lo_bits));
    crange[2 * blockIdx.x + 1] = __longlong_as_double(static_cast<long long>(hi_bits));
  }
}

// Each LP's start [x | y | s] gathered into its slots of the batch's warm region from starts that
// are already on the device (a warm-start network's output, LP k at offset k of each array).
__global__ void __launch_bounds__(kScaleThreads) k_batch_starts(const LpMeta* __restrict__ meta, double* __restrict__ warm,
                                                                DeviceStarts st, int first_lp) {
  const LpMeta& mt = meta[blockIdx.x];
  if (mt.m < 0 || mt.w_off < 0) return;
  const size_t k = static_cast<size_t>(first_lp) + blockIdx.x;
  double* w = warm + mt.w_off;
  for (int j = threadIdx.x; j < st.n; j += kScaleThreads) {
    w[j] = st.x[k * st.n + j];
    w[st.n + st.m + j] = st.s[k * st.n + j];
  }
  for (int i = threadIdx.x; i < st.m; i += kScaleThreads) w[st.n + i] = st.y[k * st.m + i];
}

// publish_iterate's scale products (interior_point.cpp:541-563) for every batched LP, one CTA per
// LP, from the final or the best iterate as the solve chose: cs*x and s/cs for the model's columns,
// rs*y for its rows. The host adds the shift (primal = shift + cs*x), so the published values are
// the ones the host arithmetic gives.
__global__ void __launch_bounds__(kScaleThreads) k_batch_publish(const LpMeta* __restrict__ meta, const LpOut* __restrict__ out,
                                                                 BatchDev d, const double* __restrict__ scl,
                                                                 long long total_n, double* __restrict__ pout) {
  const LpMeta& mt = meta[blockIdx.x];
  if (mt.m < 0) return;
  const bool best = out[blockIdx.x].use_best != 0;
  const double* x = (best ? d.bx : d.x) + mt.nv_off;
  const double* s = (best ? d.bs : d.s) + mt.nv_off;
  const double* y = (best ? d.by : d.y) + mt.mv_off;
  const double* cs = scl + mt.nv_off;
  const double* rs = scl + total_n + mt.mv_off;
  double* P = pout + mt.p_off;
  const int ns = mt.n_struct;
  for (int j = threadIdx.x; j < ns; j += kScaleThreads) {
    P[j] = __dmul_rn(cs[j], x[j]);
    P[ns + j] = __ddiv_rn(s[j], cs[j]);
  }
  for (int k = threadIdx.x; k < mt.m0; k += kScaleThreads) P[2 * ns + k] = __dmul_rn(rs[k], y[k]);
}

// SOVEREIGN_BATCH_WIDTHS="128:256,96:128,..." pins the shape of each listed bucket (by its row
// bound), so a profiler capture can run the widths an autotuned run chose; 0 when `mmax` is not
// listed or the code is not a shape
int pinned_threads(int mmax) {
  const char* e = std::getenv("SOVEREIGN_BATCH_WIDTHS");
  if (!e) return 0;
  std::istringstream in(e);
  std::string item;
  while (std::getline(in, item, ',')) {
    const size_t colon = item.find(':');
    if (colon == std::string::npos || std::atoi(item.c_str()) != mmax) continue;
    const int t = std::atoi(item.c_str() + colon + 1);
    for (int code : kShapes)
      if (t == code) return t;
  }
  return 0;
}

int threads_for(int mmax) {
  // SOVEREIGN_BATCH_THREADS=128|129|256|257|512 pins every bucket to a shape (tests run each one
  // this way; odd codes are the lean shapes)
  if (const char* e = std::getenv("SOVEREIGN_BATCH_THREADS")) {
    const int t = std::atoi(e);
    for (int code : kShapes)
      if (t == code) return t;
  }
  if (const int t = pinned_threads(mmax)) return t;
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tuned_threads.find(mmax);
  if (it != g_tuned_threads.end()) return it->second;
  (void)mmax;
  return 128;  // measured best on average without tuning (4 CTAs of 128 per SM)
}

void launch_any(const BatchDev& bd, int mmax, int code, int grid, cudaStream_t st) {
  switch (code) {
    case 128: launch_bucket<128, false>(bd, mmax, grid, st); break;
    case 129: launch_bucket<128, true>(bd, mmax, grid, st); break;
    case 257: launch_bucket<256, true>(bd, mmax, grid, st); break;
    case 512: launch_bucket<512, false>(bd, mmax, grid, st); break;
    default: launch_bucket<256, false>(bd, mmax, grid, st); break;
  }
}

// The grid of a bucket launch: every CTA that fits at once, or at most per_sm of them per SM
// (fewer resident LPs keep a bucket's per-LP vectors inside L2; the autotuner decides).
int tuned_per_sm(int mmax) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  auto it = g_tuned_per_sm.find(mmax);
  return it != g_tuned_per_sm.end() ? it->second : 0;
}

int sm_count() {
  int dev = 0, sms = 0;
  SOV_CUDA(cudaGetDevice(&dev));
  SOV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return sms;
}

int grid_for(int mmax, int code, int count, int per_sm = -1) {
  if (per_sm < 0) per_sm = tuned_per_sm(mmax);
  int cap;
  switch (code) {
    case 128: cap = max_ctas<128, false>(mmax); break;
    case 129: cap = max_ctas<128, true>(mmax); break;
    case 257: cap = max_ctas<256, true>(mmax); break;
    case 512: cap = max_ctas<512, false>(mmax); break;
    default: cap = max_ctas<256, false>(mmax); break;
  }
  if (per_sm > 0) cap = std::min(cap, per_sm * sm_count());
  return std::max(1, std::min(cap, count));
}

size_t align8(size_t v) { return (v + 7) & ~size_t(7); }

}  // namespace

Batch* batch_create(int count, const sov_model* models, const sov_options* opt_in, int opt_stride,
                    const DeviceStarts* starts, int first_lp) {
  auto model_no = [&](int i) { return std::to_string(first_lp + i); };  // the caller's numbering
  auto B = std::make_unique<Batch>();
  B->count = count;
  B->models.assign(models, models + count);
  B->forms.resize(count);
  if (opt_in) B->opt = *opt_in;
  else sov_default_lp_options(&B->opt);
  // per-LP option blocks (opt_stride bytes apart) or one shared block
  if (opt_in && opt_stride > 0) {
    B->opts.resize(count);
    for (int i = 0; i < count; ++i)
      B->opts[i] = *reinterpret_cast<const sov_options*>(reinterpret_cast<const char*>(opt_in) +
                                                         static_cast<size_t>(i) * opt_stride);
  }
  auto opt_of = [&](int i) -> const sov_options& { return B->opts.empty() ? B->opt : B->opts[i]; };
  if (starts) {
    B->has_dstarts = true;
    B->dstarts = *starts;
    B->first_lp = first_lp;
  }
  ensure_smem_limits();
  // 1. shapes, in parallel. LPs with plain columns are later built in place, straight into the
  //    pinned staging; the others get a StdForm here (build_ipm_form semantics,
  //    interior_point.cpp:224-409), batched if small enough, else solved by the single engine.
  enum : uint8_t { kInPlace = 0, kFromForm = 1, kSingle = 2 };
  std::vector<LpShape> shape(count);
  std::vector<uint8_t> kind(count);
  parallel_for(count, [&](int i) {
    LpShape sh{};
    if (plain_lp_shape(models[i], &sh) && sh.m > 0 && sh.m <= kBatchMaxRows && sh.n > 0) {
      shape[i] = sh;
      kind[i] = kInPlace;
      return;
    }
    try {
      B->forms[i] = build_std_form(models[i], false, opt_of(i).enable_scaling != 0);
    } catch (const std::exception& e) {
      throw std::runtime_error("model " + model_no(i) + ": " + e.what());
    }
    const StdForm& f = B->forms[i];
    shape[i] = LpShape{f.n_struct, f.m0, f.m, f.n, f.nnz(), 0};
    kind[i] = (f.m > 0 && f.m <= kBatchMaxRows && f.n > 0) ? kFromForm : kSingle;
  });
  // 2. offsets (serial prefix over the LPs)
  B->meta.resize(count);
  B->pub.resize(count);
  long long nnz = 0, cols = 0, rows = 0, nv = 0, mv = 0, pubn = 0, wv = 0, pv = 0;
  int from_form = 0;
  struct Run {
    long long nnz, cols, rows, mv, nv, wv;
  };
  std::vector<Run> run(count + 1);  // running totals before LP i (chunk boundaries of the staging)
  for (int i = 0; i < count; ++i) {
    run[i] = Run{nnz, cols, rows, mv, nv, wv};
    const LpShape& sh = shape[i];
    const sov_options& opt = opt_of(i);
    LpMeta& mt = B->meta[i];
    std::memset(&mt, 0, sizeof(mt));
    if (starts && (sh.n != starts->n || sh.m != starts->m))
      throw std::runtime_error("model " + model_no(i) + ": IPM form " + std::to_string(sh.m) +
                               " x " + std::to_string(sh.n) + " does not match the starts' " +
                               std::to_string(starts->m) + " x " + std::to_string(starts->n));
    if (kind[i] == kSingle) {
      B->fallback.push_back(i);
      mt.m = -1;
      continue;
    }
    mt.m = sh.m;
    mt.n = sh.n;
    mt.nnz = sh.nnz;
    mt.n_struct = sh.n_struct;
    mt.m0 = sh.m0;
    mt.scale_mode = kind[i] == kFromForm ? 2 : (opt.enable_scaling != 0 && sh.m > 0 && sh.n > 0) ? 1 : 0;
    if (kind[i] == kFromForm) ++from_form;
    mt.p_off = pv;
    pv += 2LL * sh.n_struct + sh.m0;
    mt.max_iter = opt.max_iterations;
    mt.a_off = nnz;
    mt.cp_off = cols;
    mt.rp_off = rows;
    mt.mv_off = mv;
    mt.nv_off = nv;
    mt.ftol = opt.feasibility_tol;
    mt.otol = opt.optimality_tol;
    mt.tau = opt.fraction_to_boundary;
    mt.w_off = -1;
    if (starts) {
      mt.w_off = wv;
      wv += 2LL * sh.n + sh.m;
    } else if (opt.warm_x && opt.warm_y && opt.warm_s) {
      mt.w_off = wv;
      wv += 2LL * sh.n + sh.m;
    }
    Batch::Pub& pb = B->pub[i];
    pb.n_struct = sh.n_struct;
    pb.m0 = sh.m0;
    pb.n = sh.n;
    pb.m = sh.m;
    pb.shift_off = pubn;
    pb.cs_off = pubn + sh.n_struct;
    pb.rs_off = pubn + sh.n_struct + sh.n;
    pubn += sh.n_struct + sh.n + sh.m;
    nnz += sh.nnz;
    cols += sh.n + 1;
    rows += sh.m + 1;
    nv += sh.n;
    mv += sh.m;
    // algorithmic work per iteration (roofline): vector bytes + factorization flops
    B->bytes += 6.0 * (12.0 * sh.nnz + 8.0 * (sh.m + sh.n)) + 15.0 * 8.0 * sh.n + 10.0 * 8.0 * sh.m;
    B->flops += (2.0 / 3.0) * std::pow(static_cast<double>(sh.m), 3.0);
  }
  run[count] = Run{nnz, cols, rows, mv, nv, wv};
  B->total_n = nv;
  B->total_m = mv;
  B->total_nnz = nnz;
  B->total_cols = cols;
  B->total_rows = rows;
  B->total_pub = pv;
  B->pubdata.alloc(static_cast<size_t>(std::max(1LL, pubn)));
  // buckets by m, each ordered largest-first (cost ~ m^3 + nnz); their orders travel with the inputs
  std::map<int, std::vector<int>> groups;
  for (int i = 0; i < count; ++i)
    if (B->meta[i].m > 0) groups[bucket_of(B->meta[i].m)].push_back(i);
  std::vector<double> cost(count, 0.0);
  for (int i = 0; i < count; ++i) {
    const double mm = B->meta[i].m;
    cost[i] = mm * mm * mm + 20.0 * B->meta[i].nnz;
  }
  std::vector<int> all_orders;
  all_orders.reserve(count);
  std::vector<size_t> order_at;
  for (auto it = groups.rbegin(); it != groups.rend(); ++it) {
    auto& ids = it->second;
    std::sort(ids.begin(), ids.end(), [&](int a1, int a2) { return cost[a1] > cost[a2]; });
    auto bk = std::make_unique<Batch::Bucket>();
    bk->mmax = it->first;
    bk->threads = threads_for(bk->mmax);
    bk->count = static_cast<int>(ids.size());
    bk->grid = grid_for(bk->mmax, bk->threads, bk->count);
    order_at.push_back(all_orders.size());
    all_orders.insert(all_orders.end(), ids.begin(), ids.end());
    B->buckets.push_back(std::move(bk));
  }
  // layout: meta | col_ptr | row_idx | row_ptr | col_idx | (8-aligned) cval | rval | b | c | warm | orders |
  // (8-aligned) column scales | row scales. col_idx and rval are not copied (k_batch_rows fills
  // them on the device), nor the scales, except those of LPs scaled by the host (k_batch_scale
  // computes the others)
  const size_t o_meta = 0;
  const size_t o_cp = align8(o_meta + sizeof(LpMeta) * count);
  const size_t o_ri = o_cp + sizeof(int) * cols;
  const size_t o_rp = o_ri + sizeof(int) * nnz;
  const size_t o_ci = o_rp + sizeof(int) * rows;
  const size_t o_cv = align8(o_ci + sizeof(int) * nnz);
  const size_t o_rv = o_cv + sizeof(double) * nnz;
  const size_t o_b = o_rv + sizeof(double) * nnz;
  const size_t o_c = o_b + sizeof(double) * mv;
  const size_t o_w = o_c + sizeof(double) * nv;
  const size_t o_ord = o_w + sizeof(double) * wv;
  const size_t o_scl = align8(o_ord + sizeof(int) * all_orders.size());
  const size_t total = o_scl + sizeof(double) * (nv + mv);
  B->h2d_bytes = static_cast<double>(o_ord + sizeof(int) * all_orders.size() - (sizeof(int) + sizeof(double)) * nnz);
  if (starts) B->h2d_bytes -= static_cast<double>(sizeof(double) * wv);  // gathered on the device
  B->in.alloc(total);
  B->work.alloc(static_cast<size_t>(std::max(1LL, 9 * nv + 2 * mv)));
  B->crec.alloc(static_cast<size_t>(std::max(1LL, nv)));
  B->cval2.alloc(static_cast<size_t>(std::max(1LL, nv)));
  B->out.alloc(count);
  B->nexts.alloc(std::max<size_t>(1, B->buckets.size()));
  B->pout.alloc(static_cast<size_t>(pv + 2LL * count));
  // 3. every LP's standard form written into its slots of the pinned staging, chunk by chunk in
  //    LP order; each finished chunk's slots are copied to the device (async) while the next
  //    chunk is built
  PinnedArena& arena = g_arenas[g_arena_turn.fetch_add(1) % 2];
  std::lock_guard<std::mutex> lock(arena.mu);
  unsigned char* h = arena.get(total);
  double* pubd = B->pubdata.p;
  // the copies and the input kernels on a high-priority stream: while an earlier batch's persistent
  // kernels hold the SMs, this batch's short kernels take the first slots that free up
  CudaObjectPool& pool = CudaObjectPool::get();
  cudaStream_t cs = pool.stream(true);
  B->input_stream = cs;
  auto copy_range = [&](size_t off, size_t bytes) {
    if (bytes) SOV_CUDA(cudaMemcpyAsync(B->in.p + off, h + off, bytes, cudaMemcpyHostToDevice, cs));
  };
  // chunks of the staging whose copies overlap the building of the next one (each chunk is one
  // parallel_for over the worker pool; SOVEREIGN_BATCH_CHUNKS overrides)
  int chunks = count >= 512 ? 8 : 1;
  if (const char* e = std::getenv("SOVEREIGN_BATCH_CHUNKS")) chunks = std::max(1, std::min(count, std::atoi(e)));
  try {
    for (int ch = 0; ch < chunks; ++ch) {
      const int lo = static_cast<int>(static_cast<long long>(count) * ch / chunks);
      const int hi = static_cast<int>(static_cast<long long>(count) * (ch + 1) / chunks);
      parallel_for(hi - lo, [&](int t) {
        const int i = lo + t;
        LpMeta& mt = B->meta[i];
        if (mt.m < 0) return;
        Batch::Pub& pb = B->pub[i];
        int* cp = reinterpret_cast<int*>(h + o_cp) + mt.cp_off;
        int* ri = reinterpret_cast<int*>(h + o_ri) + mt.a_off;
        int* rp = reinterpret_cast<int*>(h + o_rp) + mt.rp_off;
        int* ci = reinterpret_cast<int*>(h + o_ci) + mt.a_off;
        double* cv = reinterpret_cast<double*>(h + o_cv) + mt.a_off;
        double* rv = reinterpret_cast<double*>(h + o_rv) + mt.a_off;
        double* bb = reinterpret_cast<double*>(h + o_b) + mt.mv_off;
        double* cc = reinterpret_cast<double*>(h + o_c) + mt.nv_off;
        if (mt.w_off >= 0 && !starts) {
          const sov_options& o = opt_of(i);
          double* wd = reinterpret_cast<double*>(h + o_w) + mt.w_off;
          std::memcpy(wd, o.warm_x, sizeof(double) * mt.n);
          std::memcpy(wd + mt.n, o.warm_y, sizeof(double) * mt.m);
          std::memcpy(wd + mt.n + mt.m, o.warm_s, sizeof(double) * mt.n);
        }
        if (kind[i] == kInPlace) {
          // unscaled here; k_batch_scale scales on the device (coefficient range after: see batch_results)
          const LpFormOut out{cp, ri, cv, rp, ci, rv, bb, cc, pubd + pb.shift_off, pubd + pb.cs_off, pubd + pb.rs_off};
          try {
            build_plain_lp_into(models[i], shape[i], false, out, &pb.info, false);
          } catch (const std::exception& e) {
            throw std::runtime_error("model " + model_no(i) + ": " + e.what());
          }
          pb.info.scaling_applied = mt.scale_mode == 1;
        } else {
          const StdForm& f = B->forms[i];
          std::memcpy(cp, f.col_ptr.data(), sizeof(int) * (f.n + 1));
          std::memcpy(ri, f.row_idx.data(), sizeof(int) * f.nnz());
          std::memcpy(rp, f.row_ptr.data(), sizeof(int) * (f.m + 1));
          std::memcpy(cv, f.val.data(), sizeof(double) * f.nnz());
          std::memcpy(bb, f.b.data(), sizeof(double) * f.m);
          std::memcpy(cc, f.c.data(), sizeof(double) * f.n);
          std::copy(f.shift.begin(), f.shift.end(), pubd + pb.shift_off);
          double* hs = reinterpret_cast<double*>(h + o_scl);
          std::copy(f.col_scale.begin(), f.col_scale.end(), hs + mt.nv_off);
          std::copy(f.row_scale.begin(), f.row_scale.end(), hs + nv + mt.mv_off);
          pb.info = LpFormInfo{f.scaling_applied, f.coef_min_before, f.coef_max_before, f.coef_min_after,
                               f.coef_max_after};
        }
      });
      const Run& r0 = run[lo];
      const Run& r1 = run[hi];
      copy_range(o_cp + sizeof(int) * r0.cols, sizeof(int) * (r1.cols - r0.cols));
      copy_range(o_ri + sizeof(int) * r0.nnz, sizeof(int) * (r1.nnz - r0.nnz));
      copy_range(o_rp + sizeof(int) * r0.rows, sizeof(int) * (r1.rows - r0.rows));
      copy_range(o_cv + sizeof(double) * r0.nnz, sizeof(double) * (r1.nnz - r0.nnz));
      copy_range(o_b + sizeof(double) * r0.mv, sizeof(double) * (r1.mv - r0.mv));
      copy_range(o_c + sizeof(double) * r0.nv, sizeof(double) * (r1.nv - r0.nv));
      if (!starts) copy_range(o_w + sizeof(double) * r0.wv, sizeof(double) * (r1.wv - r0.wv));
    }
    std::memcpy(h + o_meta, B->meta.data(), sizeof(LpMeta) * count);
    if (!all_orders.empty()) std::memcpy(h + o_ord, all_orders.data(), sizeof(int) * all_orders.size());
    copy_range(o_meta, sizeof(LpMeta) * count);
    copy_range(o_ord, sizeof(int) * all_orders.size());
    if (from_form > 0)  // the scales of the LPs the host scaled
      for (int i = 0; i < count; ++i) {
        const LpMeta& mt = B->meta[i];
        if (mt.m < 0 || mt.scale_mode != 2) continue;
        copy_range(o_scl + sizeof(double) * mt.nv_off, sizeof(double) * mt.n);
        copy_range(o_scl + sizeof(double) * (nv + mt.mv_off), sizeof(double) * mt.m);
        B->h2d_bytes += sizeof(double) * (mt.n + mt.m);
      }
    arena.record(cs);  // the next user of this staging waits for these copies
    // the scaling, then the row-wise copies built on the device from the (scaled) columns
    unsigned char* din = B->in.p;
    B->scl = reinterpret_cast<double*>(din + o_scl);
    if (starts) {
      if (starts->ready) SOV_CUDA(cudaStreamWaitEvent(cs, starts->ready, 0));
      k_batch_starts<<<count, kScaleThreads, 0, cs>>>(reinterpret_cast<const LpMeta*>(din + o_meta),
                                                      reinterpret_cast<double*>(din + o_w), *starts, first_lp);
      SOV_CUDA(cudaGetLastError());
    }
    k_batch_scale<<<count, kScaleThreads, 0, cs>>>(
        reinterpret_cast<LpMeta*>(din + o_meta), reinterpret_cast<const int*>(din + o_cp),
        reinterpret_cast<const int*>(din + o_ri), reinterpret_cast<double*>(din + o_cv),
        reinterpret_cast<double*>(din + o_b), reinterpret_cast<double*>(din + o_c), B->scl, nv, B->pout.p + pv);
    SOV_CUDA(cudaGetLastError());
    k_batch_rows<<<count, kRowsThreads, 0, cs>>>(
        reinterpret_cast<const LpMeta*>(din + o_meta), reinterpret_cast<const int*>(din + o_cp),
        reinterpret_cast<const int*>(din + o_ri), reinterpret_cast<const double*>(din + o_cv),
        reinterpret_cast<const int*>(din + o_rp), reinterpret_cast<int*>(din + o_ci),
        reinterpret_cast<double*>(din + o_rv), B->crec.p, B->cval2.p);
    SOV_CUDA(cudaGetLastError());
    B->ready = pool.event(false);
    SOV_CUDA(cudaEventRecord(B->ready, cs));
    // the copies and the input kernels run on; every launch of this batch waits for `ready`
  } catch (...) {
    cudaStreamSynchronize(cs);  // `cs` goes back to the pool with the batch
    throw;
  }
  for (size_t k = 0; k < B->buckets.size(); ++k) {
    B->buckets[k]->order = reinterpret_cast<const int*>(B->in.p + o_ord) + order_at[k];
    B->buckets[k]->next = B->nexts.p + k;
  }
  BatchDev& d = B->dev;
  unsigned char* base = B->in.p;
  d.meta = reinterpret_cast<const LpMeta*>(base + o_meta);
  d.col_ptr = reinterpret_cast<const int*>(base + o_cp);
  d.row_idx = reinterpret_cast<const int*>(base + o_ri);
  d.row_ptr = reinterpret_cast<const int*>(base + o_rp);
  d.col_idx = reinterpret_cast<const int*>(base + o_ci);
  d.cval = reinterpret_cast<const double*>(base + o_cv);
  d.rval = reinterpret_cast<const double*>(base + o_rv);
  d.crec = B->crec.p;
  d.cval2 = B->cval2.p;
  d.b = reinterpret_cast<const double*>(base + o_b);
  d.c = reinterpret_cast<const double*>(base + o_c);
  d.warm = reinterpret_cast<const double*>(base + o_w);
  double* w = B->work.p;
  d.x = w;
  d.s = w + nv;
  d.dx = w + 2 * nv;
  d.ds = w + 3 * nv;
  d.dxa = w + 4 * nv;
  d.dsa = w + 5 * nv;
  d.rd = w + 6 * nv;
  d.bx = w + 7 * nv;
  d.bs = w + 8 * nv;
  d.y = w + 9 * nv;
  d.by = w + 9 * nv + mv;
  d.out = B->out.p;
  return B.release();
}

namespace {

// per-bucket streams, their join events, the fork event and the timing events, made once per batch
void make_streams(Batch* B) {
  if (B->fork) return;
  CudaObjectPool& pool = CudaObjectPool::get();
  for (size_t b = 0; b < B->buckets.size(); ++b) {
    B->streams.push_back(pool.stream(false));
    B->joins.push_back(pool.event(false));
  }
  B->fork = pool.event(false);
  B->t0 = pool.event(true);
  B->t1 = pool.event(true);
}

// fork from `from`, every bucket's counter reset and persistent launch on its own stream, join back
void enqueue_buckets(Batch* B, cudaStream_t from) {
  SOV_CUDA(cudaEventRecord(B->fork, from));
  for (size_t b = 0; b < B->buckets.size(); ++b) {
    auto& bk = B->buckets[b];
    cudaStream_t s2 = B->streams[b];
    SOV_CUDA(cudaStreamWaitEvent(s2, B->fork, 0));
    SOV_CUDA(cudaMemsetAsync(bk->next, 0, sizeof(int), s2));
    BatchDev d = B->dev;
    d.order = bk->order;
    d.count = bk->count;
    d.next = bk->next;
    launch_any(d, bk->mmax, bk->threads, bk->grid, s2);
    SOV_CUDA(cudaEventRecord(B->joins[b], s2));
    SOV_CUDA(cudaStreamWaitEvent(from, B->joins[b], 0));
  }
}

// k_batch_publish on `st` behind the solve, then the `published` event batch_results waits for
void enqueue_publish(Batch* B, cudaStream_t st) {
  if (!B->published) B->published = CudaObjectPool::get().event(false);
  const BatchDev& d = B->dev;
  k_batch_publish<<<B->count, kScaleThreads, 0, st>>>(d.meta, d.out, d, B->scl, B->total_n, B->pout.p);
  SOV_CUDA(cudaGetLastError());
  const size_t pn = static_cast<size_t>(B->total_pub + 2LL * B->count);
  B->h_out.alloc(B->count);
  B->h_pout.alloc(pn);
  SOV_CUDA(cudaMemcpyAsync(B->h_out.p, B->out.p, sizeof(LpOut) * B->count, cudaMemcpyDeviceToHost, st));
  SOV_CUDA(cudaMemcpyAsync(B->h_pout.p, B->pout.p, sizeof(double) * pn, cudaMemcpyDeviceToHost, st));
  SOV_CUDA(cudaEventRecord(B->published, st));
  B->publish_queued = true;
}

}  // namespace

// The batch's bucket launches on `st` between two timing events; batch_finish waits for them.
// Buckets run concurrently: each on its own stream forked from (and joined back into) `st`, so
// the few large LPs do not hold the SMs the smaller buckets could use. A batch solved repeatedly
// (one_shot false) has the fork / reset / launch / join sequence captured once into a CUDA graph
// and replayed; a batch solved once is launched directly (capturing and instantiating a graph
// would cost more than it saves).
void batch_launch(Batch* B, cudaStream_t st, bool one_shot) {
  make_streams(B);
  SOV_CUDA(cudaStreamWaitEvent(st, B->ready, 0));
  if (one_shot) {
    SOV_CUDA(cudaEventRecord(B->t0, st));
    enqueue_buckets(B, st);
    SOV_CUDA(cudaEventRecord(B->t1, st));
    enqueue_publish(B, st);  // read back by batch_results; outside the timed events
    return;
  }
  B->publish_queued = false;
  if (!B->graph) {
    SOV_CUDA(cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking));
    SOV_CUDA(cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal));
    enqueue_buckets(B, B->cap);
    cudaGraph_t g = nullptr;
    SOV_CUDA(cudaStreamEndCapture(B->cap, &g));
    const cudaError_t e = cudaGraphInstantiate(&B->graph, g, 0);
    cudaGraphDestroy(g);
    SOV_CUDA(e);
  }
  SOV_CUDA(cudaEventRecord(B->t0, st));
  SOV_CUDA(cudaGraphLaunch(B->graph, st));
  SOV_CUDA(cudaEventRecord(B->t1, st));
}

void batch_finish(Batch* B) {
  SOV_CUDA(cudaEventSynchronize(B->t1));
  float ms = 0.f;
  SOV_CUDA(cudaEventElapsedTime(&ms, B->t0, B->t1));
  B->launches = static_cast<int>(B->buckets.size());
  B->kernel_ms = ms;
}

void batch_solve(Batch* B, cudaStream_t st) {
  batch_launch(B, st, false);
  batch_finish(B);
}

void batch_results(Batch* B, sov_result* results) {
  const long long nv = B->total_n, mv = B->total_m, pv = B->total_pub;
  const BatchDev& d = B->dev;
  // D2H: statuses, then the published scale products of every LP and the coefficient ranges
  // (k_batch_publish picks the final or the best iterate on the device); the IPM-space iterates
  // only when a result asks for them
  if (!B->publish_queued) {
    CudaObjectPool& pool = CudaObjectPool::get();
    cudaStream_t ps = pool.stream(true);
    try {
      if (B->t1) SOV_CUDA(cudaStreamWaitEvent(ps, B->t1, 0));
      enqueue_publish(B, ps);
      SOV_CUDA(cudaStreamSynchronize(ps));
    } catch (...) {
      cudaStreamSynchronize(ps);
      pool.give_stream(ps, true);
      throw;
    }
    pool.give_stream(ps, true);
  }
  SOV_CUDA(cudaEventSynchronize(B->published));  // the publish kernel and the copies of out / pout behind it
  B->publish_queued = false;
  const LpOut* out = B->h_out.p;
  const double* hp = B->h_pout.p;
  bool want_ipm = false;
  for (int i = 0; i < B->count && !want_ipm; ++i)
    want_ipm = B->meta[i].m >= 0 && (results[i].ipm_x || results[i].ipm_s || results[i].ipm_y);
  const size_t pbytes = sizeof(double) * (pv + 2LL * B->count);
  const size_t bytes = want_ipm ? sizeof(double) * (2 * nv + mv) : 0;
  std::unique_lock<std::mutex> lock(g_arenas[0].mu, std::defer_lock);  // the iterates, when asked for
  double* h = nullptr;
  if (want_ipm) {
    lock.lock();
    h = reinterpret_cast<double*>(g_arenas[0].get(std::max<size_t>(bytes, 8)));
  }
  const double* crange = hp + pv;
  if (want_ipm && nv) SOV_CUDA(cudaMemcpy(h, d.x, sizeof(double) * 2 * nv, cudaMemcpyDeviceToHost));  // x, s adjacent
  if (want_ipm && mv) SOV_CUDA(cudaMemcpy(h + 2 * nv, d.y, sizeof(double) * mv, cudaMemcpyDeviceToHost));
  double d2h = sizeof(LpOut) * B->count + static_cast<double>(pbytes + bytes);
  std::vector<std::vector<double>> best(B->count);
  for (int i = 0; i < B->count && want_ipm; ++i) {
    const LpMeta& mt = B->meta[i];
    if (mt.m < 0 || !out[i].use_best) continue;
    best[i].resize(2 * mt.n + mt.m);
    SOV_CUDA(cudaMemcpy(best[i].data(), d.bx + mt.nv_off, sizeof(double) * mt.n, cudaMemcpyDeviceToHost));
    SOV_CUDA(cudaMemcpy(best[i].data() + mt.n, d.bs + mt.nv_off, sizeof(double) * mt.n, cudaMemcpyDeviceToHost));
    SOV_CUDA(cudaMemcpy(best[i].data() + 2 * mt.n, d.by + mt.mv_off, sizeof(double) * mt.m, cudaMemcpyDeviceToHost));
    d2h += 8.0 * (2 * mt.n + mt.m);
  }
  B->d2h_bytes = d2h;
  parallel_for(B->count, [&](int i) {
    sov_result* r = &results[i];
    const LpMeta& mt = B->meta[i];
    if (mt.m < 0) return;  // solved by the fallback path below
    const Batch::Pub& f = B->pub[i];
    const double* shift = B->pubdata.p + f.shift_off;
    const double* px = hp + mt.p_off;  // cs*x | s/cs | rs*y
    const sov_model& mdl = B->models[i];
    const LpOut& o = out[i];
    r->status = o.status;
    r->iterations = o.iterations;
    r->has_objective_value = 1;
    r->n_ipm = f.n;
    r->m_ipm = f.m;
    r->duality_gap = o.gap;
    r->primal_residual = o.p_res;
    r->dual_residual = o.d_res;
    // publish_iterate (interior_point.cpp:541-563)
    double obj = mdl.obj_constant;
    for (int j = 0; j < f.n_struct; ++j) {
      const double v = shift[j] + px[j];
      if (r->primal) r->primal[j] = v;
      obj += (mdl.obj ? mdl.obj[j] : 0.0) * v;
    }
    if (r->dual_col) std::copy(px + f.n_struct, px + 2 * f.n_struct, r->dual_col);
    if (r->dual_row) std::copy(px + 2 * f.n_struct, px + 2 * f.n_struct + f.m0, r->dual_row);
    if (want_ipm) {  // the IPM-space iterate the published values came from
      const bool use_best = o.use_best != 0;
      const double* hx = use_best ? best[i].data() : h + mt.nv_off;
      const double* hs = use_best ? best[i].data() + mt.n : h + nv + mt.nv_off;
      const double* hy = use_best ? best[i].data() + 2 * mt.n : h + 2 * nv + mt.mv_off;
      if (r->ipm_x) std::copy(hx, hx + f.n, r->ipm_x);
      if (r->ipm_s) std::copy(hs, hs + f.n, r->ipm_s);
      if (r->ipm_y) std::copy(hy, hy + f.m, r->ipm_y);
    }
    r->objective_value = obj;
    r->solve_seconds = B->kernel_ms * 1e-3;
    if (o.status == SOV_OPTIMAL)
      std::snprintf(r->message, sizeof(r->message),
                    "Optimal solution found by primal-dual interior-point (Mehrotra). Normal equations: batched "
                    "shared-memory L D L' on the GPU (%d x %d).",
                    f.m, f.m);
    else if (o.best_it)
      std::snprintf(r->message, sizeof(r->message),
                    "IPM stopped because the affine predictor factorization failed; the best iterate is returned "
                    "with optimality unproven.");
    else
      std::snprintf(r->message, sizeof(r->message),
                    "IPM stopped after %d iterations without meeting tolerance; returning best iterate from %d as a "
                    "lower-accuracy candidate. Relative duality gap = %g (tolerance %g), primal residual = %g, dual "
                    "residual = %g. Optimality is not proven.",
                    mt.max_iter, o.iterations, o.gap, mt.otol, o.p_res, o.d_res);
    if (r->diagnostics) {
      std::memset(r->diagnostics, 0, sizeof(sov_diagnostics));
      r->diagnostics->scaling_applied = f.info.scaling_applied;
      r->diagnostics->coefficient_min_abs_before = f.info.coef_min_before;
      r->diagnostics->coefficient_max_abs_before = f.info.coef_max_before;
      if (mt.scale_mode == 1) {  // range after the device scaling (+inf: no entry in range)
        const double lo = crange[2 * i];
        r->diagnostics->coefficient_min_abs_after = lo <= DBL_MAX ? lo : 0.0;
        r->diagnostics->coefficient_max_abs_after = crange[2 * i + 1];
      } else {
        r->diagnostics->coefficient_min_abs_after = f.info.coef_min_after;
        r->diagnostics->coefficient_max_abs_after = f.info.coef_max_after;
      }
      r->diagnostics->refactorizations = o.iterations + 1;
      r->diagnostics->warm_start_used = o.warm_used;
      r->diagnostics->stall_iteration = -1;
    }
  });
  // LPs the batched kernel does not take go through the single-problem engine
  for (int i : B->fallback) {
    sov_result* r = &results[i];
    const StdForm& f = B->forms[i];
    if (f.n <= 0) {
      r->status = SOV_ERROR;
      r->has_objective_value = 0;
      std::snprintf(r->message, sizeof(r->message), "IPM: empty model.");
      continue;
    }
    sov_options o = B->opts.empty() ? B->opt : B->opts[i];
    std::vector<double> wx, wy, ws;
    if (B->has_dstarts) {  // this LP's start from the device, used exactly as a host warm start
      const DeviceStarts& ds = B->dstarts;
      const size_t k = static_cast<size_t>(B->first_lp) + i;
      if (ds.ready) SOV_CUDA(cudaEventSynchronize(ds.ready));
      wx.resize(ds.n);
      wy.resize(ds.m);
      ws.resize(ds.n);
      SOV_CUDA(cudaMemcpy(wx.data(), ds.x + k * ds.n, sizeof(double) * ds.n, cudaMemcpyDeviceToHost));
      SOV_CUDA(cudaMemcpy(wy.data(), ds.y + k * ds.m, sizeof(double) * ds.m, cudaMemcpyDeviceToHost));
      SOV_CUDA(cudaMemcpy(ws.data(), ds.s + k * ds.n, sizeof(double) * ds.n, cudaMemcpyDeviceToHost));
      o.warm_x = wx.data();
      o.warm_y = wy.data();
      o.warm_s = ws.data();
    }
    cudaStream_t st;
    SOV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    try {
      solve_single(B->models[i], f, o, r, st, nullptr);
    } catch (...) {
      cudaStreamDestroy(st);
      throw;
    }
    cudaStreamDestroy(st);
  }
}

void batch_stats(const Batch* B, int* launches, double* kernel_ms, double* bytes, double* flops) {
  if (launches) *launches = B->launches;
  if (kernel_ms) *kernel_ms = B->kernel_ms;
  if (bytes) *bytes = B->bytes;
  if (flops) *flops = B->flops;
}

void batch_transfer_bytes(const Batch* B, double* h2d, double* d2h) {
  if (h2d) *h2d = B->h2d_bytes;
  if (d2h) *d2h = B->d2h_bytes;
}

void batch_destroy(Batch* B) { delete B; }

void parallel_memcpy(void* dst, const void* src, size_t bytes) {
  constexpr size_t kChunk = size_t(1) << 18;
  const int chunks = static_cast<int>((bytes + kChunk - 1) / kChunk);
  parallel_for(chunks, [&](int c) {
    const size_t off = static_cast<size_t>(c) * kChunk;
    std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, std::min(kChunk, bytes - off));
  });
}

int solve_batch(int count, const sov_model* models, const sov_options* opt, int opt_stride, sov_result* results,
                const DeviceStarts* starts) {
  if (count == 0) return SOV_OK;
  // Large batches in parts, pipelined: each part's graph is launched as soon as its inputs are on
  // the device, so the host standard form and the copies of the next part overlap the solves of the
  // ones before; the results are read back in order once all parts are launched. A part's LPs are
  // solved exactly as in one batch (per-LP work, bucket widths by m).
  // 4096 LPs per call (medians of 5-7 calls, results read back behind the solves, two stagings):
  // 4 parts 18.8-19.9 ms, 6 parts 18.4-19.2, 8 parts 18.2-18.3, 10 parts 19.5
  int parts = count >= 3072 ? 8 : count >= 2048 ? 4 : 1;
  if (const char* e = std::getenv("SOVEREIGN_BATCH_PARTS")) parts = std::max(1, std::min(count, std::atoi(e)));
  // Part sizes: equal, or (SOVEREIGN_BATCH_TAPER=1) falling linearly, part k weighted parts - k,
  // so that the last parts, whose solves nothing overlaps, are the short ones.
  bool taper = false;
  if (const char* e = std::getenv("SOVEREIGN_BATCH_TAPER")) taper = std::atoi(e) != 0;
  std::vector<int> lo_of(parts + 1);
  {
    const long long wsum = taper ? static_cast<long long>(parts) * (parts + 1) / 2 : parts;
    long long acc = 0;
    for (int k = 0; k <= parts; ++k) {
      lo_of[k] = static_cast<int>(static_cast<long long>(count) * acc / wsum);
      if (k < parts) acc += taper ? parts - k : 1;
    }
  }
  std::vector<std::unique_ptr<Batch>> batches;
  std::vector<cudaStream_t> streams;
  auto part_lo = [&](int k) { return lo_of[k]; };
  try {
    for (int k = 0; k < parts; ++k) {
      const int lo = part_lo(k), hi = part_lo(k + 1);
      if (hi == lo) {  // a tapered schedule over few LPs can leave a part empty
        batches.emplace_back(nullptr);
        continue;
      }
      const sov_options* o = (opt && opt_stride > 0)
                                 ? reinterpret_cast<const sov_options*>(reinterpret_cast<const char*>(opt) +
                                                                        static_cast<size_t>(lo) * opt_stride)
                                 : opt;
      batches.emplace_back(batch_create(hi - lo, models + lo, o, opt_stride, starts, lo));
      cudaStream_t st = CudaObjectPool::get().stream(false);
      streams.push_back(st);
      batch_launch(batches.back().get(), st, true);
    }
    for (int k = 0; k < parts; ++k) {
      if (!batches[k]) continue;
      batch_finish(batches[k].get());
      batch_results(batches[k].get(), results + part_lo(k));
    }
  } catch (...) {
    for (cudaStream_t st : streams) {
      cudaStreamSynchronize(st);
      CudaObjectPool::get().give_stream(st, false);
    }
    throw;
  }
  for (cudaStream_t st : streams) CudaObjectPool::get().give_stream(st, false);
  return SOV_OK;
}

std::string autotune(int count, const sov_model* models, const sov_options* opt, const std::string& file) {
  // Per bucket: time the bucket alone with every kernel shape (128 / 256 / 512 threads per CTA, and
  // the lean 128 / 256) and take the fastest.
  std::unique_ptr<Batch> B(batch_create(count, models, opt));
  SOV_CUDA(cudaEventSynchronize(B->ready));
  cudaStream_t st;
  SOV_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  std::vector<std::string> alone(B->buckets.size());
  std::vector<int> alone_t(B->buckets.size());
  bool any_free = false;
  for (size_t k = 0; k < B->buckets.size(); ++k) {
    auto& bk = B->buckets[k];
    if (pinned_threads(bk->mmax)) {  // threads_for gave the pinned shape: nothing to time
      alone[k] = "\"pinned\": 1";
      alone_t[k] = bk->threads;
      continue;
    }
    any_free = true;
    float best_ms = 1e30f;
    int best_t = bk->threads;
    std::ostringstream part;
    bool f2 = true;
    for (int threads : kShapes) {
      const int grid = grid_for(bk->mmax, threads, bk->count, 0);
      BatchDev d = B->dev;
      d.order = bk->order;
      d.count = bk->count;
      d.next = bk->next;
      float ms_min = 1e30f;
      for (int rep_i = 0; rep_i < 2; ++rep_i) {
        cudaEvent_t e0, e1;
        SOV_CUDA(cudaEventCreate(&e0));
        SOV_CUDA(cudaEventCreate(&e1));
        SOV_CUDA(cudaMemsetAsync(bk->next, 0, sizeof(int), st));
        SOV_CUDA(cudaEventRecord(e0, st));
        launch_any(d, bk->mmax, threads, grid, st);
        SOV_CUDA(cudaEventRecord(e1, st));
        SOV_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        SOV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        ms_min = std::min(ms_min, ms);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
      }
      part << (f2 ? "" : ", ") << "\"" << threads << "\": " << ms_min;
      f2 = false;
      if (ms_min < best_ms) {
        best_ms = ms_min;
        best_t = threads;
      }
    }
    alone[k] = part.str();
    alone_t[k] = best_t;
    bk->threads = best_t;
    bk->grid = grid_for(bk->mmax, best_t, bk->count, 0);
  }
  // Then the buckets together, as a solve runs them (concurrently, on forked streams): one pass
  // over the buckets trying each other width with the rest fixed, timing the whole step (best of
  // two); a change is kept only if the step gets at least 1 % faster.
  auto step_ms = [&]() {
    float best = 1e30f;
    for (int r = 0; r < 2; ++r) {
      batch_launch(B.get(), st, true);
      batch_finish(B.get());
      best = std::min(best, static_cast<float>(B->kernel_ms));
    }
    return best;
  };
  float cur = any_free ? step_ms() : 0.0f;
  for (auto& bk : B->buckets) {
    if (pinned_threads(bk->mmax)) continue;
    const int first_t = bk->threads;
    for (int threads : kShapes) {
      if (threads == first_t) continue;
      const int old_t = bk->threads, old_g = bk->grid;
      bk->threads = threads;
      bk->grid = grid_for(bk->mmax, threads, bk->count, 0);
      const float ms = step_ms();
      if (ms < 0.99f * cur) {
        cur = ms;
      } else {
        bk->threads = old_t;
        bk->grid = old_g;
      }
    }
  }
  // Then, per bucket with its width fixed, one resident CTA per SM fewer than fit (a smaller
  // working set of per-LP vectors for L2, the SMs' other slots left to the other buckets), kept
  // only if the whole step gets at least 1 % faster.
  std::vector<int> per_sm_kept(B->buckets.size(), 0);
  const int sms = sm_count();
  for (size_t k = 0; k < B->buckets.size(); ++k) {
    auto& bk = B->buckets[k];
    const int full = grid_for(bk->mmax, bk->threads, 1 << 30, 0) / sms;  // CTAs per SM that fit
    if (full < 2 || bk->count <= (full - 1) * sms) continue;             // nothing to trim
    const int old_g = bk->grid;
    bk->grid = grid_for(bk->mmax, bk->threads, bk->count, full - 1);
    const float ms = step_ms();
    if (ms < 0.99f * cur) {
      cur = ms;
      per_sm_kept[k] = full - 1;
    } else {
      bk->grid = old_g;
    }
  }
  SOV_CUDA(cudaStreamSynchronize(st));
  cudaStreamDestroy(st);
  // per bucket: the widths timed alone (ms), the width fastest alone, the width kept for the
  // concurrent step, its LPs; then the step time with the alone choices and with the kept ones
  std::ostringstream rep;
  rep << "{";
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    for (size_t k = 0; k < B->buckets.size(); ++k) {
      const auto& bk = B->buckets[k];
      g_tuned_threads[bk->mmax] = bk->threads;
      if (per_sm_kept[k] > 0) g_tuned_per_sm[bk->mmax] = per_sm_kept[k];
      else g_tuned_per_sm.erase(bk->mmax);
      rep << (k ? ", " : "") << "\"m<=" << bk->mmax << "\": {" << alone[k] << ", \"alone\": " << alone_t[k]
          << ", \"chosen\": " << bk->threads << ", \"per_sm\": " << per_sm_kept[k] << ", \"count\": " << bk->count
          << ", \"grid\": " << bk->grid << "}";
    }
  }
  rep << "}";
  std::string out = rep.str();
  if (!file.empty()) {
    std::ofstream o(file);
    o << out << "\n";
  }
  return out;
}

}  // namespace sov
