// band.cu -- banded LDL^T of the normal matrix in the natural row order.
//
// Used when A D A' has a small half-bandwidth kd (the convex-sequence QP: kd = 2). The elimination
// tree of a band matrix is a path, so the factorization is one dependent chain of m columns; it
// runs as a single thread with the kd x kd window of L and the last kd pivots in registers and
// the next band row prefetched, which keeps the chain to one reciprocal and O(kd^2) FMAs per
// column. Dependent rows follow the reference's tiny-pivot rule (sparse_ldlt.cpp:165-173:
// D_jj <= 1e-13 * diag -> 1e128).
#include "band.cuh"
#include "common.cuh"

namespace sov {
namespace {

// B[off * m + col] = M[col + off][col] on entry; on exit B[off * m + col] = L[col + off][col]
// (off >= 1) and dinv[col] = 1 / D[col].
template <int KD>
__global__ void k_band_ldlt(double* __restrict__ B, const double* __restrict__ diag, double* __restrict__ dinv, int m,
                            int* drop_count, int* fail) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  // win[p][q] = L[j-1-p][j-1-p-q-1]... kept as Lrow[p][q] = L[j-p][j-p-q] for p = 1..KD, q = 1..KD
  double Lrow[KD + 1][KD + 1];
  double Dprev[KD + 1];  // Dprev[p] = D[j - p]
#pragma unroll
  for (int p = 0; p <= KD; ++p) {
    Dprev[p] = 1.0;
#pragma unroll
    for (int q = 0; q <= KD; ++q) Lrow[p][q] = 0.0;
  }
  int drops = 0, bad = 0;
  double mrow[KD + 1];  // mrow[p] = M[j][j - p]
#pragma unroll
  for (int p = 0; p <= KD; ++p) mrow[p] = (p == 0 && m > 0) ? B[0] : 0.0;
  for (int j = 0; j < m; ++j) {
    // prefetch next row's band: M[j+1][j+1-p] = B[p * m + j + 1 - p]
    double next[KD + 1];
#pragma unroll
    for (int p = 0; p <= KD; ++p) next[p] = (j + 1 < m && j + 1 - p >= 0) ? B[static_cast<int64_t>(p) * m + j + 1 - p] : 0.0;
    double l[KD + 1];
    l[0] = 1.0;
#pragma unroll
    for (int p = KD; p >= 1; --p) {
      if (j - p < 0) {
        l[p] = 0.0;
        continue;
      }
      double v = mrow[p];
#pragma unroll
      for (int q = p + 1; q <= KD; ++q)
        if (j - q >= 0) v -= l[q] * Dprev[q] * Lrow[p][q - p];  // L[j][j-q] D[j-q] L[j-p][j-q]
      l[p] = v / Dprev[p];
    }
    double dj = mrow[0];
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j - p >= 0) dj -= l[p] * l[p] * Dprev[p];
    const double dref = diag[j];
    if (!isfinite(dj)) {
      bad = 1;
      dj = 1e128;
    } else if (dj <= 1e-13 * fabs(dref)) {
      dj = 1e128;
      ++drops;
    }
    // store L[j][j-p] at B[p * m + j - p], 1/D[j]
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j - p >= 0) B[static_cast<int64_t>(p) * m + j - p] = l[p];
    dinv[j] = 1.0 / dj;
    // shift windows: row j becomes "p = 1"
#pragma unroll
    for (int p = KD; p >= 2; --p) {
      Dprev[p] = Dprev[p - 1];
#pragma unroll
      for (int q = 1; q <= KD; ++q) Lrow[p][q] = Lrow[p - 1][q];
    }
    Dprev[1] = dj;
#pragma unroll
    for (int q = 1; q <= KD; ++q) Lrow[1][q] = l[q];
#pragma unroll
    for (int p = 0; p <= KD; ++p) mrow[p] = next[p];
  }
  if (drops) atomicAdd(drop_count, drops);
  if (bad) atomicExch(fail, 1);
}

template <int KD>
__global__ void k_band_solve(const double* __restrict__ B, const double* __restrict__ dinv, int m, double* __restrict__ z) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double win[KD + 1];
#pragma unroll
  for (int p = 0; p <= KD; ++p) win[p] = 0.0;
  // forward: y_j = z_j - sum_p L[j][j-p] y_{j-p}
  for (int j = 0; j < m; ++j) {
    double v = z[j];
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j - p >= 0) v -= B[static_cast<int64_t>(p) * m + j - p] * win[p];
#pragma unroll
    for (int p = KD; p >= 2; --p) win[p] = win[p - 1];
    win[1] = v;
    z[j] = v * dinv[j];
  }
  // backward: x_j = y_j / D_j - sum_p L[j+p][j] x_{j+p}
#pragma unroll
  for (int p = 0; p <= KD; ++p) win[p] = 0.0;
  for (int j = m - 1; j >= 0; --j) {
    double v = z[j];
#pragma unroll
    for (int p = 1; p <= KD; ++p)
      if (j + p < m) v -= B[static_cast<int64_t>(p) * m + j] * win[p];
#pragma unroll
    for (int p = KD; p >= 2; --p) win[p] = win[p - 1];
    win[1] = v;
    z[j] = v;
  }
}

template <int KD>
void dispatch_factor(double* B, const double* diag, double* dinv, int m, int* drops, int* fail, cudaStream_t st) {
  k_band_ldlt<KD><<<1, 1, 0, st>>>(B, diag, dinv, m, drops, fail);
}
template <int KD>
void dispatch_solve(const double* B, const double* dinv, int m, double* z, cudaStream_t st) {
  k_band_solve<KD><<<1, 1, 0, st>>>(B, dinv, m, z);
}

}  // namespace

void band_factor(const BandSystem& s, cudaStream_t st, int* launches) {
  switch (s.kd) {
    case 0: dispatch_factor<1>(s.B, s.diag, s.dinv, s.m, s.drop_count, s.fail, st); break;
    case 1: dispatch_factor<1>(s.B, s.diag, s.dinv, s.m, s.drop_count, s.fail, st); break;
    case 2: dispatch_factor<2>(s.B, s.diag, s.dinv, s.m, s.drop_count, s.fail, st); break;
    case 3: dispatch_factor<3>(s.B, s.diag, s.dinv, s.m, s.drop_count, s.fail, st); break;
    case 4: dispatch_factor<4>(s.B, s.diag, s.dinv, s.m, s.drop_count, s.fail, st); break;
    default:
      if (s.kd <= 6) dispatch_factor<6>(s.B, s.diag, s.dinv, s.m, s.drop_count, s.fail, st);
      else dispatch_factor<kBandMax>(s.B, s.diag, s.dinv, s.m, s.drop_count, s.fail, st);
  }
  SOV_LAUNCH_CHECK();
  if (launches) ++*launches;
}

void band_solve(const BandSystem& s, double* z, cudaStream_t st, int* launches) {
  switch (s.kd) {
    case 0:
    case 1: dispatch_solve<1>(s.B, s.dinv, s.m, z, st); break;
    case 2: dispatch_solve<2>(s.B, s.dinv, s.m, z, st); break;
    case 3: dispatch_solve<3>(s.B, s.dinv, s.m, z, st); break;
    case 4: dispatch_solve<4>(s.B, s.dinv, s.m, z, st); break;
    default:
      if (s.kd <= 6) dispatch_solve<6>(s.B, s.dinv, s.m, z, st);
      else dispatch_solve<kBandMax>(s.B, s.dinv, s.m, z, st);
  }
  SOV_LAUNCH_CHECK();
  if (launches) ++*launches;
}

}  // namespace sov
