// xband.cu -- Mehrotra predictor-corrector interior point for separable convex QPs with banded
// inequality rows, in x-space, with the iterate and the Newton solves in double-double.
//
// The shape: min 1/2 x'diag(q)x + c'x over free x subject to a_r x >= b_r, each row spanning at
// most kd + 1 consecutive columns (the convex-sequence QP: rows (1, -2, 1) on x_r, x_r+1, x_r+2).
// The reference reaches this shape's optimum only through its structured LISWET solvers in long
// double / __float128 (solver/qp/src/qp_interior_point.cpp:892-967 detector, :2378-2826 x-space
// pentadiagonal IPM); its generic QP IPM (:2848-3116) stalls on it, and so do FP64 normal equations:
// near the optimum the row weights z/w span more than 1e25, so Q's contribution to
// K = Q + A' diag(z/w) A vanishes below FP64 rounding of the large entries, and the multipliers z
// (up to ~1e7) leave A'z accurate only to ~1e-9. Here K is assembled, factored (banded L D L', one
// dependent chain of n columns) and solved in double-double, and x, z, the residuals b - Ax + w and
// Qx + c - A'z, and the direction's dw = A dx + rp and dz are carried in double-double too; the
// slack w, step lengths, mu and sigma stay FP64.
//
// Newton step (rows normalised to >=, slack w = Ax - b >= 0, multiplier z >= 0, theta = z / w):
//   (Q + A' theta A) dx = -rd - A'(rc / w + theta rp),   rp = Ax - w - b,  rd = Qx + c - A'z
//   dw = A dx + rp,   dz = -rc / w - theta dw
// with rc = w z for the predictor and w z + dw_aff dz_aff - sigma mu for the corrector,
// sigma = (mu_aff / mu)^3, one common step min(1, tau * max step) (Q != 0, qp_interior_point.cpp:3095),
// and the reference QP's residual and gap measures (:2975-2994): p_res = |rp|_inf / max(1, |b|_inf),
// d_res = |rd|_inf / max(1, |c|_inf + |Qx|_inf), gap = w'z / (1 + |objective|).
//
// The whole solve is one launch of one CTA: the vector passes are spread over its threads, and so
// is the banded factorization: the columns are cut into up to 512 segments, one per thread, each an
// interior factored as a band chain (window in registers, next column loaded ahead) plus a
// separator of kd columns; the separators' Schur complement, block tridiagonal, is factored by one
// thread (part_factor / part_solve below). SOVEREIGN_XBAND_SEGMENTS=1 gives the single chain.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "common.cuh"
#include "dd.cuh"
#include "xband.hpp"

namespace sov {
namespace {

constexpr int kXbThreads = 512;

struct XbOut {
  int status, iterations, history_len, failed;
  double p_res, d_res, gap, obj, mu;
  double gap_hist[SOV_HISTORY_MAX], mu_hist[SOV_HISTORY_MAX], obj_hist[SOV_HISTORY_MAX];
  double step_hist[SOV_HISTORY_MAX];
  int it_hist[SOV_HISTORY_MAX];
};

struct XbDev {
  int n, m, max_iter;
  const int *row_ptr, *col_idx, *col_ptr, *row_idx;
  const double *row_val, *col_val, *q, *c, *b;
  double obj_constant, bnorm, cnorm, feas_tol, opt_tol, tau;
  // iterates: x and z in double-double, w in FP64
  double *xh, *xl, *zh, *zl, *w;
  // work
  double *th, *rph, *rpl, *rd, *uh, *ul, *dxh, *dxl, *dw, *dzh, *dzl, *dwa, *dza;
  double *Kh, *Kl;  // (kd + 1) x n: K[j][j - p] at p * n + j, overwritten by L (p >= 1) and 1 / D (p = 0)
  // partitioned factorization: P segments, each an interior and (but the last) a separator of kd
  int P;
  double *Wh, *Wl;  // 2 kd x n: the interiors' spikes K_II^-1 K_IS (left kd columns, then right kd)
  double *Ch, *Cl;  // P x 3 x kd^2: Schur contributions of each interior (to S_{s-1}, to S_s, block (s, s-1))
  double *Th, *Tl;  // P x 2 x kd^2: separator chain factors (L_t, then D_t^-1)
  double *Rh, *Rl;  // P x 2 x kd: the interiors' contributions to the separators' right-hand sides
  XbOut* out;
};

__device__ __forceinline__ dd ld_dd(const double* h, const double* l, long long i) { return dd{h[i], l[i]}; }
__device__ __forceinline__ void st_dd(double* h, double* l, long long i, dd v) {
  h[i] = v.hi;
  l[i] = v.lo;
}

// Banded L D L' of rows [a, e) of K in place, by one thread: entries that reach left of a (the
// coupling to the separator before the range) are neither used nor overwritten. Returns false on a
// pivot that is not positive and finite (K = Q + A' theta A is positive definite, so only a
// breakdown of the iterate gives one).
template <int KD>
__device__ bool band_factor_dd(double* Kh, double* Kl, int n, int a, int e) {
  dd L[KD + 1][KD + 1];  // L[p][q] = L(j - p, j - p - q) of the rows above
  dd Dv[KD + 1];         // D(j - p)
  dd Di[KD + 1];         // 1 / D(j - p)
#pragma unroll
  for (int p = 0; p <= KD; ++p) {
    Dv[p] = dd_from(1.0);
    Di[p] = dd_from(1.0);
#pragma unroll
    for (int q = 0; q <= KD; ++q) L[p][q] = dd_from(0.0);
  }
  dd row[KD + 1];  // K(j, j - p)
#pragma unroll
  for (int p = 0; p <= KD; ++p) row[p] = (p == 0 && a < e) ? ld_dd(Kh, Kl, a) : dd_from(0.0);
  for (int j = a; j < e; ++j) {
    dd next[KD + 1];
#pragma unroll
    for (int p = 0; p <= KD; ++p)
      next[p] = (j + 1 < e && j + 1 - p >= a) ? ld_dd(Kh, Kl, static_cast<long long>(p) * n + j + 1) : dd_from(0.0);
    dd l[KD + 1];
    l[0] = dd_from(1.0);
#pragma unroll
    for (int p = KD; p >= 1; --p) {
      if (j - p < a) {
        l[p] = dd_from(0.0);
        continue;
      }
      dd v = row[p];
#pragma unroll
      for (int q = p + 1; q <= KD; ++q)  // L(j, j-q) D(j-q) L(j-p, j-q)
        if (j - q >= a) v = dd_sub(v, dd_mul(dd_mul(l[q], Dv[q]), L[p][q - p]));
      l[p] = dd_mul(v, Di[p]);
    }
    dd d = row[0];
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j - p >= a) d = dd_sub(d, dd_mul(dd_mul(l[p], l[p]), Dv[p]));
    if (!(d.hi > 0.0) || !isfinite(d.hi)) return false;
    const dd di = dd_recip(d);
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j - p >= a) st_dd(Kh, Kl, static_cast<long long>(p) * n + j, l[p]);
    st_dd(Kh, Kl, j, di);
#pragma unroll
    for (int p = KD; p >= 2; --p) {
      Dv[p] = Dv[p - 1];
      Di[p] = Di[p - 1];
#pragma unroll
      for (int q = 1; q <= KD; ++q) L[p][q] = L[p - 1][q];
    }
    Dv[1] = d;
    Di[1] = di;
#pragma unroll
    for (int q = 1; q <= KD; ++q) L[1][q] = l[q];
#pragma unroll
    for (int p = 0; p <= KD; ++p) row[p] = next[p];
  }
  return true;
}

// K_[a,e) x = rhs with the factor above, in place in rh/rl (global indexing), one thread.
template <int KD>
__device__ void band_solve_dd(const double* Kh, const double* Kl, int n, int a, int e, double* rh, double* rl) {
  dd win[KD + 1];
#pragma unroll
  for (int p = 0; p <= KD; ++p) win[p] = dd_from(0.0);
  for (int j = a; j < e; ++j) {  // L y = rhs, then y / D
    dd v = ld_dd(rh, rl, j);
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j - p >= a) v = dd_sub(v, dd_mul(ld_dd(Kh, Kl, static_cast<long long>(p) * n + j), win[p]));
#pragma unroll
    for (int p = KD; p >= 2; --p) win[p] = win[p - 1];
    win[1] = v;
    st_dd(rh, rl, j, dd_mul(v, ld_dd(Kh, Kl, j)));
  }
#pragma unroll
  for (int p = 0; p <= KD; ++p) win[p] = dd_from(0.0);
  for (int j = e - 1; j >= a; --j) {  // L' x = v
    dd v = ld_dd(rh, rl, j);
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j + p < e) v = dd_sub(v, dd_mul(ld_dd(Kh, Kl, static_cast<long long>(p) * n + j + p), win[p]));
#pragma unroll
    for (int p = KD; p >= 2; --p) win[p] = win[p - 1];
    win[1] = v;
    st_dd(rh, rl, j, v);
  }
}

// ---- partitioned factorization and solve (all threads of the CTA) ----
// Segment s of P covers [lo_s, hi_s): its interior [lo_s, e_s) with e_s = hi_s - KD, and (but the
// last) the separator S_s = [e_s, hi_s). Interiors couple only to the separators on either side,
// so with the separators ordered last K = [K_II K_IS; K_SI K_SS] has a block-diagonal K_II: every
// thread factors its own interior (band L D L'), solves for its spikes W = K_II^-1 K_IS (nonzero
// right-hand sides only next to the separators) and forms its part of the Schur complement
// S = K_SS - K_SI W, which is block tridiagonal with KD x KD blocks. Thread 0 factors S as a
// chain of P - 1 blocks. A solve runs the interiors, the separator chain and the back-substitution
// y_I - W x_S. It is the band L D L' of a symmetric permutation of K, as stable as the natural one.
template <int KD>
__device__ __forceinline__ void seg_range(int s, int P, int n, int& lo, int& e, int& hi) {
  lo = static_cast<int>(static_cast<long long>(s) * n / P);
  hi = static_cast<int>(static_cast<long long>(s + 1) * n / P);
  e = s < P - 1 ? hi - KD : hi;
}

// K(i, j), |i - j| <= KD, from the band rows; only entries the interior factors leave intact
// (separator rows, and interior entries that reach the previous separator) are read this way
template <int KD>
__device__ __forceinline__ dd k_at(const XbDev& d, int i, int j) {
  const int hi = max(i, j), p = abs(i - j);
  return ld_dd(d.Kh, d.Kl, static_cast<long long>(p) * d.n + hi);
}

template <int KD>
__device__ __forceinline__ void small_inverse(dd (&A)[KD][KD], dd (&inv)[KD][KD], bool& ok) {
#pragma unroll
  for (int r = 0; r < KD; ++r)
#pragma unroll
    for (int c = 0; c < KD; ++c) inv[r][c] = dd_from(r == c ? 1.0 : 0.0);
#pragma unroll
  for (int k = 0; k < KD; ++k) {  // Gauss-Jordan without pivoting (A is positive definite)
    if (!(A[k][k].hi > 0.0) || !isfinite(A[k][k].hi)) ok = false;
    const dd ip = dd_recip(A[k][k]);
#pragma unroll
    for (int c = 0; c < KD; ++c) {
      A[k][c] = dd_mul(A[k][c], ip);
      inv[k][c] = dd_mul(inv[k][c], ip);
    }
#pragma unroll
    for (int r = 0; r < KD; ++r) {
      if (r == k) continue;
      const dd f = A[r][k];
#pragma unroll
      for (int c = 0; c < KD; ++c) {
        A[r][c] = dd_sub(A[r][c], dd_mul(f, A[k][c]));
        inv[r][c] = dd_sub(inv[r][c], dd_mul(f, inv[k][c]));
      }
    }
  }
}

template <int KD>
__device__ void part_factor(const XbDev& d, int* bad) {
  const int P = d.P, n = d.n, s = threadIdx.x;
  constexpr int KK = KD * KD;
  if (s < P) {
    int lo, e, hi;
    seg_range<KD>(s, P, n, lo, e, hi);
    if (!band_factor_dd<KD>(d.Kh, d.Kl, n, lo, e)) {
      atomicExch(bad, 1);
    } else {
      for (int c = 0; c < 2 * KD; ++c) {  // spikes
        const bool left = c < KD;
        if ((left && s == 0) || (!left && s == P - 1)) continue;
        const int sep = left ? lo - KD + c : e + (c - KD);
        double* wh = d.Wh + static_cast<long long>(c) * n;
        double* wl = d.Wl + static_cast<long long>(c) * n;
        for (int j = lo; j < e; ++j) st_dd(wh, wl, j, abs(j - sep) <= KD ? k_at<KD>(d, j, sep) : dd_from(0.0));
        band_solve_dd<KD>(d.Kh, d.Kl, n, lo, e, wh, wl);
      }
      for (int which = 0; which < 3; ++which) {  // Schur contributions
        if ((which == 0 && s == 0) || (which == 1 && s == P - 1) || (which == 2 && (s == 0 || s == P - 1))) continue;
#pragma unroll
        for (int r = 0; r < KD; ++r) {
          const int sep = which == 0 ? lo - KD + r : e + r;
          const int j0 = which == 0 ? lo : max(lo, sep - KD), j1 = which == 0 ? min(e, sep + KD + 1) : e;
#pragma unroll
          for (int c = 0; c < KD; ++c) {
            const int col = which == 1 ? KD + c : c;
            dd acc = dd_from(0.0);
            for (int j = j0; j < j1; ++j)
              acc = dd_add(acc, dd_mul(k_at<KD>(d, sep, j), ld_dd(d.Wh + static_cast<long long>(col) * n,
                                                                  d.Wl + static_cast<long long>(col) * n, j)));
            st_dd(d.Ch, d.Cl, (static_cast<long long>(s) * 3 + which) * KK + r * KD + c, dd_neg(acc));
          }
        }
      }
    }
  }
  __syncthreads();
  // the separators' diagonal blocks A_t = K(S_t, S_t) + the Schur parts of both neighbouring
  // interiors, formed in parallel (into the slot of interior t's right contribution)
  if (s < P - 1 && !*bad) {
    int lo, e, hi;
    seg_range<KD>(s, P, n, lo, e, hi);
#pragma unroll
    for (int r = 0; r < KD; ++r)
#pragma unroll
      for (int c = 0; c < KD; ++c) {
        const long long at = (static_cast<long long>(s) * 3 + 1) * KK + r * KD + c;
        st_dd(d.Ch, d.Cl, at,
              dd_add(dd_add(k_at<KD>(d, e + r, e + c), ld_dd(d.Ch, d.Cl, at)),
                     ld_dd(d.Ch, d.Cl, (static_cast<long long>(s + 1) * 3 + 0) * KK + r * KD + c)));
      }
  }
  __syncthreads();
  if (threadIdx.x == 0 && P > 1 && !*bad) {  // block tridiagonal L D L' of S, one chain
    bool ok = true;
    dd Dprev[KD][KD], An[KD][KD], Bn[KD][KD];
#pragma unroll
    for (int r = 0; r < KD; ++r)
#pragma unroll
      for (int c = 0; c < KD; ++c) {
        An[r][c] = ld_dd(d.Ch, d.Cl, 1 * KK + r * KD + c);
        Bn[r][c] = dd_from(0.0);
      }
    for (int t = 0; t < P - 1; ++t) {
      dd A[KD][KD], B[KD][KD];
#pragma unroll
      for (int r = 0; r < KD; ++r)
#pragma unroll
        for (int c = 0; c < KD; ++c) {
          A[r][c] = An[r][c];
          B[r][c] = Bn[r][c];
        }
      if (t + 1 < P - 1)  // the next step's blocks, loaded while this one computes
#pragma unroll
        for (int r = 0; r < KD; ++r)
#pragma unroll
          for (int c = 0; c < KD; ++c) {
            An[r][c] = ld_dd(d.Ch, d.Cl, (static_cast<long long>(t + 1) * 3 + 1) * KK + r * KD + c);
            Bn[r][c] = ld_dd(d.Ch, d.Cl, (static_cast<long long>(t + 1) * 3 + 2) * KK + r * KD + c);
          }
      if (t >= 1) {
        dd L[KD][KD];
#pragma unroll
        for (int r = 0; r < KD; ++r)
#pragma unroll
          for (int c = 0; c < KD; ++c) {
            dd v = dd_from(0.0);
#pragma unroll
            for (int q = 0; q < KD; ++q) v = dd_add(v, dd_mul(B[r][q], Dprev[q][c]));
            L[r][c] = v;
            st_dd(d.Th, d.Tl, (static_cast<long long>(t) * 2 + 0) * KK + r * KD + c, v);
          }
#pragma unroll
        for (int r = 0; r < KD; ++r)
#pragma unroll
          for (int c = 0; c < KD; ++c) {
            dd v = A[r][c];
#pragma unroll
            for (int q = 0; q < KD; ++q) v = dd_sub(v, dd_mul(L[r][q], B[c][q]));
            A[r][c] = v;
          }
      }
      small_inverse<KD>(A, Dprev, ok);
#pragma unroll
      for (int r = 0; r < KD; ++r)
#pragma unroll
        for (int c = 0; c < KD; ++c) st_dd(d.Th, d.Tl, (static_cast<long long>(t) * 2 + 1) * KK + r * KD + c, Dprev[r][c]);
    }
    if (!ok) atomicExch(bad, 1);
  }
  __syncthreads();
}

// K x = rhs in place in xh/xl with the partitioned factor.
template <int KD>
__device__ void part_solve(const XbDev& d, double* xh, double* xl) {
  const int P = d.P, n = d.n, s = threadIdx.x;
  constexpr int KK = KD * KD;
  if (s < P) {
    int lo, e, hi;
    seg_range<KD>(s, P, n, lo, e, hi);
    band_solve_dd<KD>(d.Kh, d.Kl, n, lo, e, xh, xl);  // y_I
#pragma unroll
    for (int side = 0; side < 2; ++side) {  // K(S, I_s) y_I onto S_{s-1} (side 0) and S_s (side 1)
      if ((side == 0 && s == 0) || (side == 1 && s == P - 1)) continue;
#pragma unroll
      for (int r = 0; r < KD; ++r) {
        const int sep = side == 0 ? lo - KD + r : e + r;
        const int j0 = side == 0 ? lo : max(lo, sep - KD), j1 = side == 0 ? min(e, sep + KD + 1) : e;
        dd acc = dd_from(0.0);
        for (int j = j0; j < j1; ++j) acc = dd_add(acc, dd_mul(k_at<KD>(d, sep, j), ld_dd(xh, xl, j)));
        st_dd(d.Rh, d.Rl, (static_cast<long long>(s) * 2 + side) * KD + r, acc);
      }
    }
  }
  __syncthreads();
  // separators' right-hand sides less the interiors' contributions, in parallel
  if (s < P - 1) {
    int lo, e, hi;
    seg_range<KD>(s, P, n, lo, e, hi);
#pragma unroll
    for (int r = 0; r < KD; ++r)
      st_dd(xh, xl, e + r,
            dd_sub(dd_sub(ld_dd(xh, xl, e + r), ld_dd(d.Rh, d.Rl, (static_cast<long long>(s) * 2 + 1) * KD + r)),
                   ld_dd(d.Rh, d.Rl, (static_cast<long long>(s + 1) * 2 + 0) * KD + r)));
  }
  __syncthreads();
  if (threadIdx.x == 0 && P > 1) {  // forward chain z_t = r_t - L_t z_{t-1}, in the separator slots
    dd z[KD], rn[KD], Ln[KD][KD];
    {
      int lo, e, hi;
      seg_range<KD>(0, P, n, lo, e, hi);
#pragma unroll
      for (int r = 0; r < KD; ++r) z[r] = ld_dd(xh, xl, e + r);  // z_0 = r_0
    }
    for (int t = 1; t < P - 1; ++t) {
      int lo, e, hi;
      seg_range<KD>(t, P, n, lo, e, hi);
#pragma unroll
      for (int r = 0; r < KD; ++r) {
        rn[r] = ld_dd(xh, xl, e + r);
#pragma unroll
        for (int c = 0; c < KD; ++c) Ln[r][c] = ld_dd(d.Th, d.Tl, (static_cast<long long>(t) * 2 + 0) * KK + r * KD + c);
      }
      dd zn[KD];
#pragma unroll
      for (int r = 0; r < KD; ++r) {
        dd v = rn[r];
#pragma unroll
        for (int c = 0; c < KD; ++c) v = dd_sub(v, dd_mul(Ln[r][c], z[c]));
        zn[r] = v;
      }
#pragma unroll
      for (int r = 0; r < KD; ++r) {
        z[r] = zn[r];
        st_dd(xh, xl, e + r, zn[r]);
      }
    }
  }
  __syncthreads();
  if (s < P - 1) {  // w_t = D_t^-1 z_t, in parallel
    int lo, e, hi;
    seg_range<KD>(s, P, n, lo, e, hi);
    dd z[KD];
#pragma unroll
    for (int c = 0; c < KD; ++c) z[c] = ld_dd(xh, xl, e + c);
#pragma unroll
    for (int r = 0; r < KD; ++r) {
      dd v = dd_from(0.0);
#pragma unroll
      for (int c = 0; c < KD; ++c) v = dd_add(v, dd_mul(ld_dd(d.Th, d.Tl, (static_cast<long long>(s) * 2 + 1) * KK + r * KD + c), z[c]));
      st_dd(xh, xl, e + r, v);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && P > 2) {  // backward chain x_t = w_t - L_{t+1}' x_{t+1}
    dd xn[KD];
    {
      int lo, e, hi;
      seg_range<KD>(P - 2, P, n, lo, e, hi);
#pragma unroll
      for (int r = 0; r < KD; ++r) xn[r] = ld_dd(xh, xl, e + r);
    }
    for (int t = P - 3; t >= 0; --t) {
      int lo, e, hi;
      seg_range<KD>(t, P, n, lo, e, hi);
      dd w[KD], Lt[KD][KD];
#pragma unroll
      for (int r = 0; r < KD; ++r) {
        w[r] = ld_dd(xh, xl, e + r);
#pragma unroll
        for (int c = 0; c < KD; ++c) Lt[r][c] = ld_dd(d.Th, d.Tl, (static_cast<long long>(t + 1) * 2 + 0) * KK + c * KD + r);
      }
#pragma unroll
      for (int r = 0; r < KD; ++r)
#pragma unroll
        for (int c = 0; c < KD; ++c) w[r] = dd_sub(w[r], dd_mul(Lt[r][c], xn[c]));
#pragma unroll
      for (int r = 0; r < KD; ++r) {
        st_dd(xh, xl, e + r, w[r]);
        xn[r] = w[r];
      }
    }
  }
  __syncthreads();
  if (s < P && P > 1) {  // x_I = y_I - W_left x_S(s-1) - W_right x_S(s)
    int lo, e, hi;
    seg_range<KD>(s, P, n, lo, e, hi);
    dd xs[2 * KD];
#pragma unroll
    for (int c = 0; c < 2 * KD; ++c) {
      const bool left = c < KD;
      xs[c] = ((left && s == 0) || (!left && s == P - 1)) ? dd_from(0.0) : ld_dd(xh, xl, left ? lo - KD + c : e + (c - KD));
    }
    for (int j = lo; j < e; ++j) {
      dd v = ld_dd(xh, xl, j);
#pragma unroll
      for (int c = 0; c < 2 * KD; ++c)
        if (xs[c].hi != 0.0 || xs[c].lo != 0.0)
          v = dd_sub(v, dd_mul(ld_dd(d.Wh + static_cast<long long>(c) * n, d.Wl + static_cast<long long>(c) * n, j), xs[c]));
      st_dd(xh, xl, j, v);
    }
  }
  __syncthreads();
}

// (A v)_r in double-double
__device__ __forceinline__ dd row_dot(const XbDev& d, int r, const double* vh, const double* vl) {
  dd s = dd_from(0.0);
  for (int e = d.row_ptr[r]; e < d.row_ptr[r + 1]; ++e) s = dd_add(s, dd_mul_d(ld_dd(vh, vl, d.col_idx[e]), d.row_val[e]));
  return s;
}

// (A' u)_j in double-double
__device__ __forceinline__ dd col_dot(const XbDev& d, int j, const double* uh, const double* ul) {
  dd s = dd_from(0.0);
  for (int e = d.col_ptr[j]; e < d.col_ptr[j + 1]; ++e) s = dd_add(s, dd_mul_d(ld_dd(uh, ul, d.row_idx[e]), d.col_val[e]));
  return s;
}

template <int KD>
__global__ void __launch_bounds__(kXbThreads, 1) k_xband_ipm(XbDev d) {
  __shared__ double red[4 * 32];
  __shared__ double s_mu, s_sigma, s_alpha_p, s_alpha_d;
  __shared__ int s_stop, s_bad;
  const int tid = threadIdx.x;
  const int n = d.n, m = d.m;
  const double inf = INFINITY;
  // the reference QP stops at its tolerances; this path goes two decades further (cheap in
  // double-double) so that its objective meets the exact structured answer to 1e-8
  const double ftol = d.feas_tol * 1e-2, otol = d.opt_tol * 1e-2;
  int it = 0;
  for (;; ++it) {
    // ---- residuals, mu, objective ----
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // max |rp|, max |rd|, max |Qx|, w'z
    for (int r = tid; r < m; r += kXbThreads) {
      const dd rp = dd_add_d(dd_add_d(row_dot(d, r, d.xh, d.xl), -d.w[r]), -d.b[r]);
      st_dd(d.rph, d.rpl, r, rp);
      v[0] = fmax(v[0], fabs(rp.hi));
      v[3] += d.w[r] * d.zh[r];
    }
    double objp = 0.0;
    for (int j = tid; j < n; j += kXbThreads) {
      const dd qx = dd_mul_d(ld_dd(d.xh, d.xl, j), d.q[j]);
      const dd rd = dd_sub(dd_add_d(qx, d.c[j]), col_dot(d, j, d.zh, d.zl));
      d.rd[j] = rd.hi;
      v[1] = fmax(v[1], fabs(rd.hi));
      v[2] = fmax(v[2], fabs(qx.hi));
      objp += d.c[j] * d.xh[j] + 0.5 * d.q[j] * d.xh[j] * d.xh[j];
    }
    const int ops4[4] = {1, 1, 1, 0};
    block_reduce<4>(v, ops4, red);
    double o1[1] = {objp};
    const int ops1[1] = {0};
    block_reduce<1>(o1, ops1, red);
    if (tid == 0) {
      const double mu = v[3] / m;
      const double obj = o1[0] + d.obj_constant;
      const double p_res = v[0] / d.bnorm;
      const double d_res = v[1] / fmax(1.0, d.cnorm + v[2]);
      const double gap = v[3] / (1.0 + fabs(obj));
      XbOut* o = d.out;
      o->p_res = p_res;
      o->d_res = d_res;
      o->gap = gap;
      o->obj = obj;
      o->mu = mu;
      o->iterations = it;
      if (o->history_len < SOV_HISTORY_MAX) {
        const int h = o->history_len++;
        o->it_hist[h] = it;
        o->gap_hist[h] = gap;
        o->mu_hist[h] = mu;
        o->obj_hist[h] = obj;
      }
      s_mu = mu;
      s_stop = 0;
      if (!isfinite(mu) || !isfinite(p_res) || !isfinite(d_res)) {
        o->status = SOV_ERROR;
        o->failed = 1;
        s_stop = 1;
      } else if (p_res <= ftol && d_res <= ftol && gap <= otol) {
        o->status = SOV_OPTIMAL;
        s_stop = 1;
      } else if (it >= d.max_iter) {
        // at the limit the reference QP's own tolerances decide; otherwise ERROR without an
        // objective, as its failure exits publish (qp_interior_point.cpp:3042-3048, :3112-3115)
        o->status = (p_res <= d.feas_tol && d_res <= d.feas_tol && gap <= d.opt_tol) ? SOV_OPTIMAL : SOV_ERROR;
        s_stop = 1;
      }
    }
    __syncthreads();
    if (s_stop) break;
    // ---- K = Q + A' theta A, double-double ----
    for (int r = tid; r < m; r += kXbThreads) d.th[r] = d.zh[r] / d.w[r];
    __syncthreads();
    for (int j = tid; j < n; j += kXbThreads) {
      dd acc[KD + 1];
#pragma unroll
      for (int p = 0; p <= KD; ++p) acc[p] = dd_from(0.0);
      acc[0] = dd_from(d.q[j]);
      for (int e = d.col_ptr[j]; e < d.col_ptr[j + 1]; ++e) {
        const int r = d.row_idx[e];
        const double a = d.col_val[e], t = d.th[r];
        for (int f = d.row_ptr[r]; f < d.row_ptr[r + 1]; ++f) {
          const int k = d.col_idx[f];
          const int p = j - k;
          if (p < 0 || p > KD) continue;
          const dd prod = dd_mul_d(two_prod(a, d.row_val[f]), t);
#pragma unroll
          for (int q = 0; q <= KD; ++q)
            if (q == p) acc[q] = dd_add(acc[q], prod);
        }
      }
#pragma unroll
      for (int p = 0; p <= KD; ++p) st_dd(d.Kh, d.Kl, static_cast<long long>(p) * n + j, acc[p]);
    }
    __syncthreads();
    if (tid == 0) s_bad = 0;
    __syncthreads();
    part_factor<KD>(d, &s_bad);
    if (tid == 0 && s_bad) {
      d.out->status = SOV_ERROR;
      d.out->failed = 2;
      s_stop = 1;
    }
    __syncthreads();
    if (s_stop) break;
    // ---- predictor (pass 0) and corrector (pass 1) ----
    for (int pass = 0; pass < 2; ++pass) {
      const double mu = s_mu, sigma = pass ? s_sigma : 0.0;
      // u = rc / w + theta rp
      for (int r = tid; r < m; r += kXbThreads) {
        const double rc = d.w[r] * d.zh[r] + (pass ? d.dwa[r] * d.dza[r] - sigma * mu : 0.0);
        st_dd(d.uh, d.ul, r, dd_add_d(dd_mul_d(ld_dd(d.rph, d.rpl, r), d.th[r]), rc / d.w[r]));
      }
      __syncthreads();
      // rhs = -rd - A'u (into dx, solved in place)
      for (int j = tid; j < n; j += kXbThreads)
        st_dd(d.dxh, d.dxl, j, dd_neg(dd_add_d(col_dot(d, j, d.uh, d.ul), d.rd[j])));
      __syncthreads();
      part_solve<KD>(d, d.dxh, d.dxl);
      // dw = A dx + rp, dz = -rc / w - theta dw; largest steps to the boundary
      double a[2] = {inf, inf};
      for (int r = tid; r < m; r += kXbThreads) {
        const double rc = d.w[r] * d.zh[r] + (pass ? d.dwa[r] * d.dza[r] - sigma * mu : 0.0);
        const dd dwv = dd_add(row_dot(d, r, d.dxh, d.dxl), ld_dd(d.rph, d.rpl, r));
        const dd dzv = dd_neg(dd_add_d(dd_mul_d(dwv, d.th[r]), rc / d.w[r]));
        d.dw[r] = dwv.hi;
        st_dd(d.dzh, d.dzl, r, dzv);
        if (dwv.hi < 0.0) a[0] = fmin(a[0], -d.w[r] / dwv.hi);
        if (dzv.hi < 0.0) a[1] = fmin(a[1], -d.zh[r] / dzv.hi);
      }
      const int ops2[2] = {2, 2};
      block_reduce<2>(a, ops2, red);
      if (tid == 0) {
        s_alpha_p = fmin(1.0, a[0]);
        s_alpha_d = fmin(1.0, a[1]);
      }
      __syncthreads();
      if (pass == 0) {
        // mu_aff and sigma = (mu_aff / mu)^3 (qp_interior_point.cpp, as interior_point.cpp:666-673)
        const double ap = s_alpha_p, ad = s_alpha_d;
        double ma[1] = {0.0};
        for (int r = tid; r < m; r += kXbThreads) {
          d.dwa[r] = d.dw[r];
          d.dza[r] = d.dzh[r];
          ma[0] += (d.w[r] + ap * d.dw[r]) * (d.zh[r] + ad * d.dzh[r]);
        }
        block_reduce<1>(ma, ops1, red);
        if (tid == 0) {
          const double ratio = (ma[0] / m) / mu;
          s_sigma = fmin(1.0, ratio * ratio * ratio);
        }
        __syncthreads();
      }
    }
    // ---- common step ----
    const double alpha = fmin(1.0, d.tau * fmin(s_alpha_p, s_alpha_d));
    for (int j = tid; j < n; j += kXbThreads)
      st_dd(d.xh, d.xl, j, dd_add(ld_dd(d.xh, d.xl, j), dd_mul_d(ld_dd(d.dxh, d.dxl, j), alpha)));
    for (int r = tid; r < m; r += kXbThreads) {
      d.w[r] += alpha * d.dw[r];
      st_dd(d.zh, d.zl, r, dd_add(ld_dd(d.zh, d.zl, r), dd_mul_d(ld_dd(d.dzh, d.dzl, r), alpha)));
    }
    if (tid == 0 && it < SOV_HISTORY_MAX) d.out->step_hist[it] = alpha;
    __syncthreads();
  }
}

// Starting point: x = -Q^-1 c (the unconstrained minimiser), slack w = Ax - b shifted into the
// interior (by 1.5 times its most negative entry), z = 1, then both shifted by half the
// complementarity over the other's sum so that the products w_r z_r start balanced (Mehrotra's
// recipe, Mehrotra 1992, section 7).
__global__ void k_xband_start(XbDev d) {
  // one CTA: the shift needs the minimum of w and the sums
  __shared__ double red[4 * 32];
  __shared__ double s_shift, s_dw, s_dz;
  const int tid = threadIdx.x, n = d.n, m = d.m;
  for (int j = tid; j < n; j += blockDim.x) {
    d.xh[j] = -d.c[j] / d.q[j];
    d.xl[j] = 0.0;
  }
  __syncthreads();
  double v[1] = {INFINITY};
  for (int r = tid; r < m; r += blockDim.x) {
    const dd wr = dd_add_d(row_dot(d, r, d.xh, d.xl), -d.b[r]);
    d.w[r] = wr.hi;
    v[0] = fmin(v[0], wr.hi);
  }
  const int opmin[1] = {2};
  block_reduce<1>(v, opmin, red);
  if (tid == 0) s_shift = fmax(-1.5 * v[0], 0.0);
  __syncthreads();
  double s[3] = {0.0, 0.0, 0.0};  // w'z, sum w, sum z
  for (int r = tid; r < m; r += blockDim.x) {
    d.w[r] += s_shift;
    s[0] += d.w[r];
    s[1] += d.w[r];
    s[2] += 1.0;
  }
  const int opsum[3] = {0, 0, 0};
  block_reduce<3>(s, opsum, red);
  if (tid == 0) {
    const bool flat = !(s[0] > 0.0);  // the unconstrained minimiser sits on every row's boundary
    s_dw = flat ? 1.0 : 0.5 * s[0] / s[2];
    s_dz = flat ? 1.0 : 0.5 * s[0] / s[1];
  }
  __syncthreads();
  for (int r = tid; r < m; r += blockDim.x) {
    d.w[r] += s_dw;
    d.zh[r] = 1.0 + s_dz;
    d.zl[r] = 0.0;
  }
}

template <class T>
struct XbBuf {
  T* p = nullptr;
  cudaStream_t st = nullptr;
  XbBuf(size_t count, cudaStream_t s) : st(s) {
    SOV_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), sizeof(T) * std::max<size_t>(count, 1), st));
  }
  ~XbBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  XbBuf(const XbBuf&) = delete;
  XbBuf& operator=(const XbBuf&) = delete;
  void put(const std::vector<T>& h) {
    if (!h.empty()) SOV_CUDA(cudaMemcpyAsync(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st));
  }
};

}  // namespace

bool xband_prepare(const sov_model& p, XBandModel* out) {
  if (const char* off = std::getenv("SOVEREIGN_QP_DISABLE"))
    if ((std::string(",") + off + ",").find(",xband,") != std::string::npos) return false;
  const int n = p.n, m = p.m;
  if (!p.q_col_ptr || p.maximize || n < 1 || m < 1) return false;
  XBandModel& x = *out;
  x = XBandModel{};
  x.n = n;
  x.m = m;
  x.q.assign(n, 0.0);
  for (int j = 0; j < n; ++j)
    for (int k = p.q_col_ptr[j]; k < p.q_col_ptr[j + 1]; ++k) {
      if (p.q_row_idx[k] != j) return false;  // a coupling term
      x.q[j] += p.q_values[k];
    }
  for (int j = 0; j < n; ++j) {
    if (!(x.q[j] > 0.0) || !std::isfinite(x.q[j])) return false;
    if (p.lb && p.lb[j] > -1e29) return false;  // only free variables
    if (p.ub && p.ub[j] < 1e29) return false;
  }
  x.row_sign.resize(m);
  for (int i = 0; i < m; ++i) {
    if (p.sense[i] == SOV_EQ) return false;
    x.row_sign[i] = p.sense[i] == SOV_GE ? 1 : -1;
  }
  // rows: sum duplicates, span check
  std::vector<std::vector<std::pair<int, double>>> rows(m);
  for (int j = 0; j < n; ++j)
    for (int k = p.col_ptr[j]; k < p.col_ptr[j + 1]; ++k) {
      auto& row = rows[p.row_idx[k]];
      const double v = x.row_sign[p.row_idx[k]] * p.values[k];
      if (!row.empty() && row.back().first == j) row.back().second += v;
      else row.push_back({j, v});
    }
  int kd = 0;
  for (int i = 0; i < m; ++i) {
    if (rows[i].empty()) continue;
    kd = std::max(kd, rows[i].back().first - rows[i].front().first);
    if (kd > kXBandMaxKd) return false;
  }
  x.kd = std::max(1, kd);
  x.row_ptr.assign(m + 1, 0);
  for (int i = 0; i < m; ++i) {
    for (const auto& e : rows[i]) {
      x.col_idx.push_back(e.first);
      x.row_val.push_back(e.second);
    }
    x.row_ptr[i + 1] = static_cast<int32_t>(x.col_idx.size());
  }
  x.col_ptr.assign(n + 1, 0);
  for (int i = 0; i < m; ++i)
    for (const auto& e : rows[i]) x.col_ptr[e.first + 1]++;
  for (int j = 0; j < n; ++j) x.col_ptr[j + 1] += x.col_ptr[j];
  x.row_idx.resize(x.col_idx.size());
  x.col_val.resize(x.col_idx.size());
  {
    std::vector<int32_t> at(x.col_ptr.begin(), x.col_ptr.end() - 1);
    for (int i = 0; i < m; ++i)
      for (const auto& e : rows[i]) {
        x.row_idx[at[e.first]] = i;
        x.col_val[at[e.first]++] = e.second;
      }
  }
  x.c.assign(n, 0.0);
  for (int j = 0; j < n; ++j) x.c[j] = p.obj ? p.obj[j] : 0.0;
  x.b.resize(m);
  for (int i = 0; i < m; ++i) x.b[i] = x.row_sign[i] * p.rhs[i];
  x.obj_constant = p.obj_constant;
  return true;
}

int solve_xband(const sov_model& model, const XBandModel& xb, const sov_options& opt, sov_result* r,
                cudaStream_t st, EngineStats* stats) {
  const int n = xb.n, m = xb.m, kd = xb.kd;
  const size_t nnz = xb.col_idx.size();
  XbBuf<int32_t> row_ptr(m + 1, st), col_idx(nnz, st), col_ptr(n + 1, st), row_idx(nnz, st);
  XbBuf<double> row_val(nnz, st), col_val(nnz, st), q(n, st), c(n, st), b(m, st);
  row_ptr.put(xb.row_ptr);
  col_idx.put(xb.col_idx);
  col_ptr.put(xb.col_ptr);
  row_idx.put(xb.row_idx);
  row_val.put(xb.row_val);
  col_val.put(xb.col_val);
  q.put(xb.q);
  c.put(xb.c);
  b.put(xb.b);
  // n-vectors: xh xl rd dxh dxl; m-vectors: zh zl w th rph rpl uh ul dw dzh dzl dwa dza; band 2 (kd+1) n
  // segments of the partitioned factorization: one per thread, at least 16 kd columns each
  int P = std::max(1, std::min(kXbThreads, n / (16 * kd)));
  if (const char* e = std::getenv("SOVEREIGN_XBAND_SEGMENTS")) P = std::max(1, std::min(P, std::atoi(e)));
  const size_t nv = 5, mv = 13, kk = static_cast<size_t>(kd) * kd;
  const size_t part = 2 * (2 * static_cast<size_t>(kd) * n + 3 * P * kk + 2 * P * kk + 2 * static_cast<size_t>(P) * kd);
  XbBuf<double> work(nv * n + mv * m + 2 * static_cast<size_t>(kd + 1) * n + part, st);
  XbBuf<XbOut> out(1, st);
  SOV_CUDA(cudaMemsetAsync(out.p, 0, sizeof(XbOut), st));
  XbDev d{};
  d.n = n;
  d.m = m;
  d.max_iter = std::max(1, opt.max_iterations);
  d.row_ptr = row_ptr.p;
  d.col_idx = col_idx.p;
  d.col_ptr = col_ptr.p;
  d.row_idx = row_idx.p;
  d.row_val = row_val.p;
  d.col_val = col_val.p;
  d.q = q.p;
  d.c = c.p;
  d.b = b.p;
  d.obj_constant = xb.obj_constant;
  double bn = 0.0, cn = 0.0;
  for (double v : xb.b) bn = std::max(bn, std::fabs(v));
  for (double v : xb.c) cn = std::max(cn, std::fabs(v));
  d.bnorm = std::max(1.0, bn);
  d.cnorm = std::max(1.0, cn);  // the slack columns' zero costs do not change max |c|
  d.feas_tol = opt.feasibility_tol;
  d.opt_tol = opt.optimality_tol;
  d.tau = opt.fraction_to_boundary;
  double* wp = work.p;
  auto take = [&wp](size_t count) {
    double* q0 = wp;
    wp += count;
    return q0;
  };
  d.xh = take(n);
  d.xl = take(n);
  d.rd = take(n);
  d.dxh = take(n);
  d.dxl = take(n);
  d.zh = take(m);
  d.zl = take(m);
  d.w = take(m);
  d.th = take(m);
  d.rph = take(m);
  d.rpl = take(m);
  d.uh = take(m);
  d.ul = take(m);
  d.dw = take(m);
  d.dzh = take(m);
  d.dzl = take(m);
  d.dwa = take(m);
  d.dza = take(m);
  d.Kh = take(static_cast<size_t>(kd + 1) * n);
  d.Kl = take(static_cast<size_t>(kd + 1) * n);
  d.P = P;
  d.Wh = take(2 * static_cast<size_t>(kd) * n);
  d.Wl = take(2 * static_cast<size_t>(kd) * n);
  d.Ch = take(3 * P * kk);
  d.Cl = take(3 * P * kk);
  d.Th = take(2 * P * kk);
  d.Tl = take(2 * P * kk);
  d.Rh = take(2 * static_cast<size_t>(P) * kd);
  d.Rl = take(2 * static_cast<size_t>(P) * kd);
  d.out = out.p;
  cudaEvent_t e0, e1;
  SOV_CUDA(cudaEventCreate(&e0));
  SOV_CUDA(cudaEventCreate(&e1));
  SOV_CUDA(cudaEventRecord(e0, st));
  k_xband_start<<<1, kXbThreads, 0, st>>>(d);
  switch (kd) {
    case 1: k_xband_ipm<1><<<1, kXbThreads, 0, st>>>(d); break;
    case 2: k_xband_ipm<2><<<1, kXbThreads, 0, st>>>(d); break;
    case 3: k_xband_ipm<3><<<1, kXbThreads, 0, st>>>(d); break;
    default: k_xband_ipm<4><<<1, kXbThreads, 0, st>>>(d); break;
  }
  SOV_LAUNCH_CHECK();
  SOV_CUDA(cudaEventRecord(e1, st));
  XbOut o;
  std::vector<double> x(n), z(m);
  SOV_CUDA(cudaMemcpyAsync(&o, out.p, sizeof(XbOut), cudaMemcpyDeviceToHost, st));
  SOV_CUDA(cudaMemcpyAsync(x.data(), d.xh, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  SOV_CUDA(cudaMemcpyAsync(z.data(), d.zh, sizeof(double) * m, cudaMemcpyDeviceToHost, st));
  SOV_CUDA(cudaStreamSynchronize(st));
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (stats) {
    stats->launches += 2;
    stats->factorizations += o.iterations;
    stats->kernel_ms += ms;
  }
  r->status = o.status;
  r->iterations = o.iterations;
  r->has_objective_value = o.status == SOV_OPTIMAL ? 1 : 0;
  r->duality_gap = o.gap;
  r->primal_residual = o.p_res;
  r->dual_residual = o.d_res;
  r->n_ipm = n + m;
  r->m_ipm = m;
  r->solve_seconds = ms * 1e-3;
  double obj = model.obj_constant;
  for (int j = 0; j < n; ++j) obj += xb.c[j] * x[j] + 0.5 * xb.q[j] * x[j] * x[j];
  r->objective_value = obj;
  if (r->primal) std::copy(x.begin(), x.end(), r->primal);
  if (r->dual_col) std::fill(r->dual_col, r->dual_col + n, 0.0);  // free columns carry no bound multiplier
  if (r->dual_row)
    for (int i = 0; i < m; ++i) r->dual_row[i] = xb.row_sign[i] * z[i];
  if (sov_diagnostics* g = r->diagnostics) {
    std::memset(g, 0, sizeof(*g));
    g->structured_qp = 1;
    g->refactorizations = o.iterations;
    g->history_len = o.history_len;
    for (int h = 0; h < o.history_len; ++h) {
      g->history_iterations[h] = o.it_hist[h];
      g->gap_history[h] = o.gap_hist[h];
      g->mu_history[h] = o.mu_hist[h];
      g->objective_history[h] = o.obj_hist[h];
    }
    g->step_history_len = std::min(o.iterations, SOV_HISTORY_MAX);
    for (int h = 0; h < g->step_history_len; ++h) g->primal_step_history[h] = g->dual_step_history[h] = o.step_hist[h];
    g->stall_iteration = -1;
  }
  char desc[200];
  std::snprintf(desc, sizeof desc,
                "x-space Q + A'ZW^-1A, banded LDL^T in double-double on the GPU (order %d, half-bandwidth %d)", n, kd);
  std::string msg;
  if (o.status == SOV_OPTIMAL)
    msg = std::string("Optimal convex QP found by Mehrotra predictor-corrector IPM. KKT system: normal equations, ") +
          desc + ".";
  else if (o.failed)
    msg = std::string("QP-IPM Newton factorization failed (") + desc + ").";
  else
    msg = std::string("QP-IPM iteration limit reached without convergence (") + desc + ").";
  std::snprintf(r->message, sizeof(r->message), "%s", msg.c_str());
  return SOV_OK;
}

}  // namespace sov
