// dense.cu -- dense normal-matrix path on the GPU.
//
// Assembly: one gather pass over a precomputed contribution map (no atomics, deterministic).
// Factorization: blocked right-looking Cholesky, 64-wide panels; one CTA factors a diagonal block
// in shared memory and inverts it, the panel below is L_ik = A_ik L_kk^-T (a GEMM with the
// inverse), and the trailing lower triangle gets A_ij -= L_ik L_jk^T. One launch per panel does
// both as flag-ordered work items, the next diagonal block's factor among them (look-ahead).
// Solves: dataflow triangular solves, one cooperative launch per direction; row block i waits
// (acquire flag, bounded spin) for the blocks it depends on, so the off-diagonal GEMV work of all
// blocks overlaps and only the 64x64 diagonal products sit on the critical path.
#include <cooperative_groups.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <stdexcept>

#include "common.cuh"
#include "dense.cuh"

namespace sov {

template <class T>
__device__ __forceinline__ T big_pivot();
template <>
__device__ __forceinline__ double big_pivot<double>() {
  return kBigPivotD;
}
template <>
__device__ __forceinline__ float big_pivot<float>() {
  return kBigPivotF;
}

__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }
__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
// four consecutive elements from 16-byte-aligned shared memory
__device__ __forceinline__ void load4(const double* p, double v[4]) {
  const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}
__device__ __forceinline__ void load4(const float* p, float v[4]) {
  const float4 a = *reinterpret_cast<const float4*>(p);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = a.z;
  v[3] = a.w;
}
// sixteen consecutive elements from 16-byte-aligned global memory, widened to double
__device__ __forceinline__ void load16(const double* p, double v[16]) {
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double2 a = reinterpret_cast<const double2*>(p)[k];
    v[2 * k] = a.x;
    v[2 * k + 1] = a.y;
  }
}
__device__ __forceinline__ void load16(const float* p, double v[16]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float4 a = reinterpret_cast<const float4*>(p)[k];
    v[4 * k] = a.x;
    v[4 * k + 1] = a.y;
    v[4 * k + 2] = a.z;
    v[4 * k + 3] = a.w;
  }
}

__device__ __forceinline__ double column_weight(int mode, int k, const double* x, const double* s,
                                                const double* qdiag, const uint8_t* free_col) {
  if (mode == kWeightOnes) return 1.0;
  const double xk = fmax(x[k], 1e-16), sk = fmax(s[k], 1e-16);
  if (mode == kWeightLp) return xk / sk;
  if (mode == kWeightTheta) return sk / xk;
  const double h = free_col[k] ? 0.0 : sk / xk;
  return 1.0 / (qdiag[k] + h);
}

// layout_ld > 0: dense column-major with that leading dimension; layout_ld < 0: band storage
// with -layout_ld = m (diagonal offset major).
template <class T>
__global__ void k_assemble(AssemblyDev am, const double* __restrict__ x, const double* __restrict__ s,
                           const double* __restrict__ qdiag, const uint8_t* __restrict__ free_col, int mode,
                           double reg, T* __restrict__ out, double* __restrict__ diag_out, int m, int layout_ld) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= am.ntargets) return;
  double acc = 0.0;
  for (int p = am.ptr[t]; p < am.ptr[t + 1]; ++p)
    acc += am.w[p] * column_weight(mode, am.col[p], x, s, qdiag, free_col);
  const int64_t tg = am.target[t];
  int row = -1;
  if (layout_ld > 0) {
    const int r = static_cast<int>(tg % layout_ld), c = static_cast<int>(tg / layout_ld);
    if (r == c) row = r;
  } else if (tg < m) {
    row = static_cast<int>(tg);
  }
  if (row >= 0) {
    acc += reg;
    diag_out[row] = acc;
  }
  out[tg] = static_cast<T>(acc);
}

template <class T>
void launch_assemble(const AssemblyDev& am, const double* x, const double* s, const double* qdiag,
                     const uint8_t* free_col, int mode, double reg, T* out, double* diag_out, int m,
                     int layout_ld, cudaStream_t st) {
  if (am.ntargets == 0) return;
  k_assemble<T><<<ceil_div(am.ntargets, 256), 256, 0, st>>>(am, x, s, qdiag, free_col, mode, reg, out, diag_out, m,
                                                           layout_ld);
  SOV_LAUNCH_CHECK();
}

template <class T>
__global__ void k_pad_identity(T* M, int m, int mp) {
  const int i = m + blockIdx.x * blockDim.x + threadIdx.x;
  if (i < mp) M[static_cast<int64_t>(i) * mp + i] = T(1);
}

template <class T>
void launch_dense_clear(T* M, int m, int mp, cudaStream_t st) {
  SOV_CUDA(cudaMemsetAsync(M, 0, sizeof(T) * static_cast<size_t>(mp) * mp, st));
  if (mp > m) {
    k_pad_identity<T><<<ceil_div(mp - m, 128), 128, 0, st>>>(M, m, mp);
    SOV_LAUNCH_CHECK();
  }
}

// ---------------------------------------------------------------------------------------------
// Diagonal block (64 x 64) on 256 threads, right-looking over 8-column panels with look-ahead (one
// barrier per panel), then the blocked inverse of the 64 x 64 factor. Pivots come from one
// reciprocal square root (l_jj = p * rsqrt(p)), whose reciprocal is kept for the panel solves and
// the inverse.
// ---------------------------------------------------------------------------------------------
constexpr int kPanel = 8;
// diagonal factor's shared memory: A and I (64 x 65 each) and two transposed panels (8 x 64 each)
template <class T>
constexpr size_t potrf_smem_bytes() {
  return sizeof(T) * (2 * kNB * (kNB + 1) + 2 * kPanel * kNB);
}

template <int kId, int kCount>
__device__ __forceinline__ void bar_sync() {
  asm volatile("bar.sync %0, %1;" ::"n"(kId), "n"(kCount) : "memory");
}

// Row block p (rows 8p..8p+7) of X = L^-1, into I, once L's rows 8p..8p+7 are final in A and the
// earlier row blocks of X are in I, in three steps:
//   x1  X_pp = L_pp^-1, one column per thread (eight threads), by forward substitution;
//   x2  T_pj = sum_{k=j}^{8p-1} L[8p+q][k] X[k][j] for every column j < 8p, one entry at a time
//       from a shared counter, so threads join as they come free; T goes to X's place;
//   x3  X_pj = -X_pp T_pj, one entry per thread, written after a barrier (in place of T).
template <class T>
__device__ __forceinline__ void inverse_x1(const T (*A)[kNB + 1], T (*I)[kNB + 1], const T* rinv, int p, int c) {
  // L_pp x = e_c, right-looking with every index static (x starts as e_c, so the entries above c
  // stay zero)
  const int R = p * kPanel;
  T l[kPanel * (kPanel - 1) / 2], ri[kPanel], x[kPanel];
#pragma unroll
  for (int r = 0; r < kPanel; ++r) {
    ri[r] = rinv[R + r];
    x[r] = r == c ? T(1) : T(0);
#pragma unroll
    for (int k = 0; k < r; ++k) l[r * (r - 1) / 2 + k] = A[R + r][R + k];
  }
#pragma unroll
  for (int k = 0; k < kPanel; ++k) {
    x[k] *= ri[k];
#pragma unroll
    for (int r = k + 1; r < kPanel; ++r) x[r] -= l[r * (r - 1) / 2 + k] * x[k];
  }
#pragma unroll
  for (int r = 0; r < kPanel; ++r) I[R + r][R + c] = x[r];
}

template <class T>
__device__ __forceinline__ void inverse_x2(const T (*A)[kNB + 1], T (*I)[kNB + 1], int p, int* next) {
  const int R = p * kPanel;
  for (int e = atomicAdd(next, 1); e < kPanel * R; e = atomicAdd(next, 1)) {
    const int q = e % kPanel, j = e / kPanel;
    // by 8-row blocks of X from j's own (X is lower triangular: rows above j in it are zero),
    // each block's 16 loads issued together
    T a0 = T(0), a1 = T(0);
    for (int k0 = j & ~(kPanel - 1); k0 < R; k0 += kPanel) {
      T l[kPanel], x[kPanel];
#pragma unroll
      for (int t = 0; t < kPanel; ++t) {
        l[t] = A[R + q][k0 + t];
        x[t] = I[k0 + t][j];
      }
#pragma unroll
      for (int t = 0; t < kPanel; t += 2) {
        a0 += l[t] * x[t];
        a1 += l[t + 1] * x[t + 1];
      }
    }
    I[R + q][j] = a0 + a1;
  }
}

// kThreads threads from u = 0, on barrier kBar; every 8p * 8 <= 2 * kThreads
template <int kThreads, int kBar, class T>
__device__ __forceinline__ void inverse_x3(T (*I)[kNB + 1], int p, int u) {
  const int R = p * kPanel;
  T x[2];
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const int e = u + v * kThreads;
    if (e < kPanel * R) {
      const int q = e % kPanel, j = e / kPanel;
      T acc = T(0);
#pragma unroll
      for (int r = 0; r < kPanel; ++r)
        if (r <= q) acc += I[R + q][R + r] * I[R + r][j];
      x[v] = -acc;
    }
  }
  bar_sync<kBar, kThreads>();
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    const int e = u + v * kThreads;
    if (e < kPanel * R) I[R + e % kPanel][e / kPanel] = x[v];
  }
}

// One 8-column panel of the diagonal block on the 64 threads of warps 0-1: every one of them
// factors the 8 x 8 diagonal block (rows/cols k0..k0+7 of A) in registers with the same
// arithmetic (no exchange on the pivot chain, the pivot rule without branches); then (after
// barrier 2, where warps 2-7 signal that the rows below are updated, if kWaitRows) the thread
// with a row below (row k0 + 8 + tid) solves it against that factor and stores it to A and,
// transposed, to Lw (Lw[c][i] = L[i][k0 + c]). Warps 0 and 1 store halves of the factored 8 x 8
// block and the pivot reciprocals.
template <bool kWaitRows, class T>
__device__ __forceinline__ void factor_panel(T (*A)[kNB + 1], T (*Lw)[kNB], T* rinv, const double* dref, int k0,
                                             int r0, int m, double drop_tol, int& drops, int& bad) {
  const int tid = threadIdx.x;
  const bool has_row = tid < kNB - k0 - kPanel;
  T d[kPanel][kPanel], dinv[kPanel];
  double thr[kPanel];
#pragma unroll
  for (int j = 0; j < kPanel; ++j) {
    thr[j] = drop_tol * dref[k0 + j];
#pragma unroll
    for (int c = 0; c <= j; ++c) d[j][c] = A[k0 + j][k0 + c];
  }
#pragma unroll
  for (int j = 0; j < kPanel; ++j) {
    const T p = d[j][j];
    const double pd = static_cast<double>(p);
    // dependent row (sparse_ldlt.cpp:165-173): pivot not finite, or at most tol * |diag|
    const bool finite = fabs(pd) <= DBL_MAX;
    const bool drop = !(finite && pd > thr[j]);
    bad |= !finite;
    drops += (drop && r0 + k0 + j < m);
    const T inv_p = rsqrt_t(p);
    const T inv = drop ? T(1) / big_pivot<T>() : inv_p;
    d[j][j] = drop ? big_pivot<T>() : p * inv_p;
    dinv[j] = inv;
#pragma unroll
    for (int q = j + 1; q < kPanel; ++q) d[q][j] *= inv;
#pragma unroll
    for (int q = j + 1; q < kPanel; ++q)
#pragma unroll
      for (int k = j + 1; k <= q; ++k) d[q][k] -= d[q][j] * d[k][j];
  }
  if (kWaitRows) asm volatile("bar.sync 2, 256;" ::: "memory");
  if (has_row) {
    const int i = k0 + kPanel + tid;
    T r[kPanel];
#pragma unroll
    for (int c = 0; c < kPanel; ++c) r[c] = A[i][k0 + c];
#pragma unroll
    for (int c = 0; c < kPanel; ++c) {
      r[c] *= dinv[c];
#pragma unroll
      for (int e = c + 1; e < kPanel; ++e) r[e] -= r[c] * d[e][c];
    }
#pragma unroll
    for (int c = 0; c < kPanel; ++c) {
      A[i][k0 + c] = r[c];
      Lw[c][i] = r[c];
    }
  }
  if (tid == 0) {
#pragma unroll
    for (int q = 0; q < kPanel / 2; ++q) {
      rinv[k0 + q] = dinv[q];
#pragma unroll
      for (int c = 0; c <= q; ++c) A[k0 + q][k0 + c] = d[q][c];
    }
  } else if (tid == 32) {
#pragma unroll
    for (int q = kPanel / 2; q < kPanel; ++q) {
      rinv[k0 + q] = dinv[q];
#pragma unroll
      for (int c = 0; c <= q; ++c) A[k0 + q][k0 + c] = d[q][c];
    }
  }
}

// The diagonal block's lower triangle from M into A (upper entries zero); 256 threads.
template <class T>
__device__ __forceinline__ void potrf_load(const T* __restrict__ M, int ld, int kb, unsigned char* potrf_raw) {
  T(*A)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(potrf_raw);
  const int tid = threadIdx.x, r0 = kb * kNB;
#pragma unroll
  for (int h = 0; h < 2; ++h) {  // 8 loads in flight per thread
    T v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = tid + 256 * (8 * h + u), c = idx / kNB, r = idx % kNB;
      v[u] = r >= c ? M[static_cast<int64_t>(r0 + c) * ld + r0 + r] : T(0);
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = tid + 256 * (8 * h + u);
      A[idx % kNB][idx / kNB] = v[u];
    }
  }
}

// Factor and invert the diagonal block held in A (the first 64 x 65 elements of `potrf_raw`,
// lower triangle, upper entries zero); stores L to M and L^-1 to Linv. Runs on a CTA of 256
// threads; `potrf_raw` is potrf_smem_bytes<T>() of dynamic shared memory.
// Panels with look-ahead: while warps 0-1 apply panel p's update to panel p+1's diagonal block and
// factor it, warps 2-7 apply panel p's update to the rows below it (handed over on a barrier the
// row solves wait on) and then to the trailing triangle right of panel p+1, so each panel costs
// one block-wide barrier and the longer of the two chains. Warps 2-7 then also compute row block p
// of the inverse (rows of L up to panel p are final), so only the last row block follows the
// panels.
template <class T>
__device__ void potrf_core(T* __restrict__ M, int ld, int kb, const double* __restrict__ diag, int m,
                           T* __restrict__ Linv, int* drop_count, int* fail, double drop_tol,
                           unsigned char* potrf_raw) {
  T(*A)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(potrf_raw);
  T(*I)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(potrf_raw + sizeof(T) * kNB * (kNB + 1));
  __shared__ T rinv[kNB];
  __shared__ double dref[kNB];
  __shared__ int x2_next[kNB / kPanel];  // per row block of the inverse: next entry of its x2 step
  const int tid = threadIdx.x;
  const int r0 = kb * kNB;
  if (tid < kNB) dref[tid] = r0 + tid < m ? fabs(diag[r0 + tid]) : 1.0;
  if (tid < kNB / kPanel) x2_next[tid] = 0;
  __syncthreads();
  int drops = 0, bad = 0;
  // two panels' columns below their diagonal blocks, transposed (Lt[c][i] = L[i][k0 + c]), so an
  // update reads consecutive rows per vector load
  T(*Lt0)[kNB] = reinterpret_cast<T(*)[kNB]>(potrf_raw + 2 * sizeof(T) * kNB * (kNB + 1));
  T(*Lt1)[kNB] = Lt0 + kPanel;
  // warps 2-7: 4 x 4 tile (ti, tj) of the trailing update, u = ti (ti + 1) / 2 + tj, the same for
  // every panel (a triangle of nt tile rows uses u below nt (nt + 1) / 2)
  const int u = tid - kNB;
  int ti = 0, tj = 0;
  if (u >= 0) {
    ti = static_cast<int>((sqrtf(8.0f * u + 1.0f) - 1.0f) * 0.5f);
    while (ti * (ti + 1) / 2 > u) --ti;
    while ((ti + 1) * (ti + 2) / 2 <= u) ++ti;
    tj = u - ti * (ti + 1) / 2;
  }
  if (tid < kNB) factor_panel<false, T>(A, Lt0, rinv, dref, 0, r0, m, drop_tol, drops, bad);
  __syncthreads();
  for (int p = 0; p + 1 < kNB / kPanel; ++p) {
    const int K0 = (p + 1) * kPanel, K1 = K0 + kPanel;  // panel p+1's first column, and the next
    T(*Lc)[kNB] = (p & 1) ? Lt1 : Lt0;                 // panel p
    T(*Ln)[kNB] = (p & 1) ? Lt0 : Lt1;                 // panel p + 1
    if (tid < kNB) {
      // panel p's update of panel p+1's diagonal block, one entry per thread, shared through A
      if (tid < kPanel * (kPanel + 1) / 2) {
        int q = 0;
        while ((q + 1) * (q + 2) / 2 <= tid) ++q;
        const int c = tid - q * (q + 1) / 2;
        T a = A[K0 + q][K0 + c];
#pragma unroll
        for (int k = 0; k < kPanel; ++k) a -= Lc[k][K0 + q] * Lc[k][K0 + c];
        A[K0 + q][K0 + c] = a;
      }
      asm volatile("bar.sync 1, 64;" ::: "memory");  // warps 0-1: the diagonal block is updated
      factor_panel<true, T>(A, Ln, rinv, dref, K0, r0, m, drop_tol, drops, bad);
    } else {
      // panel p's update of panel p+1's columns below its diagonal block (two entries per
      // thread), signalled to warps 0-1 on barrier 2 without waiting
      {
        const int i = K1 + (u >> 2), c0 = (u & 3) * 2;
        if (i < kNB) {
          T li[kPanel];
#pragma unroll
          for (int k = 0; k < kPanel; ++k) li[k] = Lc[k][i];
#pragma unroll
          for (int c = c0; c < c0 + 2; ++c) {
            T a = A[i][K0 + c];
#pragma unroll
            for (int k = 0; k < kPanel; ++k) a -= li[k] * Lc[k][K0 + c];
            A[i][K0 + c] = a;
          }
        }
      }
      asm volatile("bar.arrive 2, 256;" ::: "memory");
      // row block p of the inverse: x1 on threads that have no tiles, x2 shared by all
      if (u >= 88 && u < 88 + kPanel) inverse_x1<T>(A, I, rinv, p, u - 88);
      // panel p's update of the trailing triangle (rows and columns from K1)
      const int nt = (kNB - K1) / 4;
      if (ti < nt) {
        const int i0 = K1 + 4 * ti, j0 = K1 + 4 * tj;
        T acc[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int v = 0; v < 4; ++v) acc[q][v] = A[i0 + q][j0 + v];
#pragma unroll
        for (int k = 0; k < kPanel; ++k) {
          T li[4], lj[4];
          load4(&Lc[k][i0], li);
          load4(&Lc[k][j0], lj);
#pragma unroll
          for (int q = 0; q < 4; ++q)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[q][v] -= li[q] * lj[v];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
#pragma unroll
          for (int v = 0; v < 4; ++v)
            if (j0 + v <= i0 + q) A[i0 + q][j0 + v] = acc[q][v];
      }
      inverse_x2<T>(A, I, p, &x2_next[p]);
      if (p > 0) {
        bar_sync<3, 192>();
        inverse_x3<192, 3, T>(I, p, u);
      }
    }
    __syncthreads();
  }
  // the inverse's last row block, on all threads
  constexpr int kLast = kNB / kPanel - 1;
  if (tid >= 256 - kPanel) inverse_x1<T>(A, I, rinv, kLast, tid - (256 - kPanel));
  inverse_x2<T>(A, I, kLast, &x2_next[kLast]);
  __syncthreads();
  inverse_x3<256, 0, T>(I, kLast, tid);
  __syncthreads();
#pragma unroll 8
  for (int v = 0; v < kNB * kNB / 256; ++v) {
    const int idx = tid + 256 * v, cc = idx / kNB, r = idx % kNB;
    if (r >= cc) M[static_cast<int64_t>(r0 + cc) * ld + r0 + r] = A[r][cc];
    Linv[static_cast<int64_t>(kb) * kNB * kNB + idx] = r >= cc ? I[r][cc] : T(0);
  }
  if (tid == 0) {
    if (drops) atomicAdd(drop_count, drops);
    if (bad) atomicExch(fail, 1);
  }
}

template <class T>
__device__ __forceinline__ void potrf_block(T* __restrict__ M, int ld, int kb, const double* __restrict__ diag, int m,
                                            T* __restrict__ Linv, int* drop_count, int* fail, double drop_tol,
                                            unsigned char* potrf_raw) {
  potrf_load<T>(M, ld, kb, potrf_raw);
  potrf_core<T>(M, ld, kb, diag, m, Linv, drop_count, fail, drop_tol, potrf_raw);
}

template <class T>
__global__ void __launch_bounds__(256) k_potrf_diag(T* __restrict__ M, int ld, int kb, const double* __restrict__ diag,
                                                    int m, T* __restrict__ Linv, int* drop_count, int* fail,
                                                    double drop_tol, unsigned* tickets) {
  extern __shared__ __align__(16) unsigned char potrf_raw[];
  if (tickets != nullptr && threadIdx.x == 0) *tickets = 0u;
  potrf_block<T>(M, ld, kb, diag, m, Linv, drop_count, fail, drop_tol, potrf_raw);
}

// acc[p][q] += sum_k Xs[k][tx + 16 p] Ys[k][ty + 16 q], tx = tid % 16, ty = tid / 16 (256 threads):
// a half-warp reads 16 consecutive entries of Xs (one wavefront) and one entry of Ys (broadcast),
// and its results are 16 consecutive rows of a column-major tile (coalesced stores)
template <class T>
__device__ __forceinline__ void tile_nt(const T (*Xs)[kNB], const T (*Ys)[kNB], T (&acc)[4][4]) {
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll 8
  for (int k = 0; k < kNB; ++k) {
    T a[4], b[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      a[q] = Xs[k][tx + 16 * q];
      b[q] = Ys[k][ty + 16 * q];
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[p][q] += a[p] * b[q];
  }
}

// Two 64 x 64 slices into shared memory, dst[k][r] = src[k * ld + r], on 256 threads with 16
// loads in flight per thread; kBypassL1 reads past L1 (data written by other CTAs of this launch).
template <bool kBypassL1, class T>
__device__ __forceinline__ void load_slices(T (*Xs)[kNB], const T* __restrict__ xsrc, int64_t xld, T (*Ys)[kNB],
                                            const T* __restrict__ ysrc, int64_t yld) {
  const int tid = threadIdx.x;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    T vx[8], vy[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = tid + 256 * (8 * h + u), k = idx / kNB, r = idx % kNB;
      vx[u] = kBypassL1 ? __ldcg(xsrc + k * xld + r) : xsrc[k * xld + r];
      vy[u] = kBypassL1 ? __ldcg(ysrc + k * yld + r) : ysrc[k * yld + r];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = tid + 256 * (8 * h + u);
      Xs[idx / kNB][idx % kNB] = vx[u];
      Ys[idx / kNB][idx % kNB] = vy[u];
    }
  }
}

constexpr long long kSpinLimit = 1ll << 22;  // bounded wait (x >= 64 ns per poll -> > 0.25 s)

__device__ __forceinline__ bool wait_flag(const unsigned* flag, unsigned epoch) {
  long long n = 0;
  while (ld_acquire(flag) != epoch) {
    if (++n > kSpinLimit) return false;
    __nanosleep(64);
  }
  return true;
}

__device__ __forceinline__ void tile_triangle(int t, int& ii, int& jj) {
  // t -> (ii, jj) with 0 <= jj <= ii, t = ii (ii + 1) / 2 + jj
  ii = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((ii + 1) * (ii + 2) / 2 <= t) ++ii;
  while (ii * (ii + 1) / 2 > t) --ii;
  jj = t - ii * (ii + 1) / 2;
}

// One launch per panel kb < nb - 1: the panel solves L_ik = A_ik Linv_kk^T of the R = nb - kb - 1
// row blocks below it and the trailing updates A_ij -= L_ik L_jk^T of the tiles kb < j <= i, as
// R + R (R + 1) / 2 - 1 work items taken in ticket order (an atomic counter):
//   item 0      the look-ahead chain: row block kb + 1's panel solve, then its diagonal tile's
//               update from the solved block still in shared memory, then the factor and inverse
//               of that diagonal block (potrf_block), so the next panel's diagonal factor starts
//               as soon as its own inputs exist rather than after the whole panel;
//   1 .. R-1    the other panel solves, each publishing its row block with a release flag;
//   R ..        the other trailing tiles, each waiting (acquire, bounded) for its two row blocks.
// A trailing tile only waits for panel solves, which never wait and hold lower tickets, so every
// item it waits for was taken by a CTA that is already running. Blocks solved by other CTAs of
// the launch are read past L1 (ld.global.cg).
template <class T>
__global__ void __launch_bounds__(256) k_panel_update(T* __restrict__ M, int ld, int kb, int nb,
                                                      const double* __restrict__ diag, int m, T* __restrict__ Linv,
                                                      int* drop_count, int* fail, double drop_tol, unsigned* flags,
                                                      unsigned stamp, unsigned* tickets, unsigned base) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*Xs)[kNB] = reinterpret_cast<T(*)[kNB]>(smem_raw);
  T(*Ys)[kNB] = reinterpret_cast<T(*)[kNB]>(smem_raw + sizeof(T) * kNB * kNB);
  __shared__ unsigned item_s;
  __shared__ int ok_s;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  if (tid == 0) item_s = atomicAdd(tickets, 1u) - base;
  __syncthreads();
  const int item = static_cast<int>(item_s);
  const int R = nb - kb - 1, k0 = kb * kNB;
  if (item < R) {
    const int i = kb + 1 + item, r0 = i * kNB;
    // Ys[k][c] = Linv[c][k] = Lk[k * 64 + c]
    load_slices<false>(Xs, M + static_cast<int64_t>(k0) * ld + r0, ld, Ys, Linv + static_cast<int64_t>(kb) * kNB * kNB,
                       kNB);
    __syncthreads();
    T acc[4][4] = {};
    tile_nt<T>(Xs, Ys, acc);
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int p = 0; p < 4; ++p) M[static_cast<int64_t>(k0 + ty + 16 * q) * ld + r0 + tx + 16 * p] = acc[p][q];
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      st_release(flags + i, stamp);
    }
    if (item != 0) return;
    // look-ahead: A_ii - L_ik L_ik^T from the block just solved, straight into the diagonal
    // factor's shared-memory tile, then its factor and inverse
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int p = 0; p < 4; ++p) Xs[ty + 16 * q][tx + 16 * p] = acc[p][q];
    T cur[4][4];  // the diagonal tile's lower triangle, loaded while the product runs
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int r = tx + 16 * p, c = ty + 16 * q;
        cur[p][q] = r >= c ? M[static_cast<int64_t>(r0 + c) * ld + r0 + r] : T(0);
      }
    __syncthreads();
    T upd[4][4] = {};
    tile_nt<T>(Xs, Xs, upd);
    __syncthreads();  // Xs, which the factor's tile overlays, is fully read
    T(*A)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(smem_raw);
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int p = 0; p < 4; ++p) {
        const int r = tx + 16 * p, c = ty + 16 * q;
        A[r][c] = r >= c ? cur[p][q] - upd[p][q] : T(0);
      }
    potrf_core<T>(M, ld, kb + 1, diag, m, Linv, drop_count, fail, drop_tol, smem_raw);
    return;
  }
  int ii, jj;
  tile_triangle(item - R + 1, ii, jj);
  const int i = kb + 1 + ii, j = kb + 1 + jj;
  if (tid == 0) ok_s = wait_flag(flags + i, stamp) && wait_flag(flags + j, stamp);
  __syncthreads();
  if (!ok_s) {
    if (tid == 0) atomicExch(fail, 1);
    return;
  }
  const int r0 = i * kNB, c0 = j * kNB;
  load_slices<true>(Xs, M + static_cast<int64_t>(k0) * ld + r0, ld, Ys, M + static_cast<int64_t>(k0) * ld + c0, ld);
  __syncthreads();
  T acc[4][4] = {};
  tile_nt<T>(Xs, Ys, acc);
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int p = 0; p < 4; ++p) M[static_cast<int64_t>(c0 + ty + 16 * q) * ld + r0 + tx + 16 * p] -= acc[p][q];
}

template <class T>
void dense_potrf_block(const DenseSystem<T>& s, int kb, cudaStream_t st) {
  const size_t smem_potrf = potrf_smem_bytes<T>();
  once_per_device((const void*)k_potrf_diag<T>, [&] {
    SOV_CUDA(cudaFuncSetAttribute(k_potrf_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_potrf));
  });
  k_potrf_diag<T><<<1, 256, smem_potrf, st>>>(s.M, s.mp, kb, s.diag, s.m, s.Linv, s.drop_count, s.fail, s.drop_tol,
                                              nullptr);
}

// panel stamps: top bit set, so they never equal a triangular-solve epoch on the same flags;
// a generation per factorization and the panel index below it
constexpr int kStampPanelBits = 11;
std::atomic<unsigned> g_factor_generation{0};

template <class T>
void dense_cholesky(const DenseSystem<T>& s, cudaStream_t st, int* launches) {
  const size_t smem_potrf = potrf_smem_bytes<T>();
  once_per_device((const void*)k_panel_update<T>, [&] {
    SOV_CUDA(cudaFuncSetAttribute(k_potrf_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_potrf));
    SOV_CUDA(cudaFuncSetAttribute(k_panel_update<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_potrf));
  });
  if (s.nb >= (1 << kStampPanelBits)) throw std::runtime_error("dense factor: too many row blocks");
  const unsigned gen = (g_factor_generation.fetch_add(1) & ((1u << (31 - kStampPanelBits)) - 1)) << kStampPanelBits;
  // panel 0's diagonal block alone (it also resets the ticket counter); every later one is
  // factored by item 0 of the previous panel's launch
  k_potrf_diag<T><<<1, 256, smem_potrf, st>>>(s.M, s.mp, 0, s.diag, s.m, s.Linv, s.drop_count, s.fail, s.drop_tol,
                                              s.tickets);
  int n = 1;
  unsigned base = 0;
  for (int kb = 0; kb + 1 < s.nb; ++kb) {
    const int R = s.nb - kb - 1;
    const int items = R + R * (R + 1) / 2 - 1;
    const unsigned stamp = 0x80000000u | gen | static_cast<unsigned>(kb);
    k_panel_update<T><<<items, 256, smem_potrf, st>>>(s.M, s.mp, kb, s.nb, s.diag, s.m, s.Linv, s.drop_count, s.fail,
                                                       s.drop_tol, s.flags, stamp, s.tickets, base);
    base += static_cast<unsigned>(items);
    ++n;
  }
  SOV_LAUNCH_CHECK();
  if (launches) *launches += n;
}

// ---------------------------------------------------------------------------------------------
// Dataflow triangular solves
// ---------------------------------------------------------------------------------------------
constexpr int kSolveBatch = 8;  // dependencies a triangular-solve block takes per flag check

// Warp 0: how many consecutive flags first, first + step, ... (at most n <= 32) are released,
// waiting (bounded) until the first one is; 0 when the wait gives up.
__device__ __forceinline__ int released_run(const unsigned* flags, int first, int step, int n, unsigned epoch) {
  const int lane = threadIdx.x & 31;
  long long spins = 0;
  for (;;) {
    const bool ready = lane < n && ld_acquire(flags + first + step * lane) == epoch;
    const unsigned mask = __ballot_sync(kFull, ready);
    const int run = __ffs(~mask) - 1;
    if (run > 0) return run;
    if (++spins > kSpinLimit) return 0;
    __nanosleep(64);
  }
}

// Forward: L y = r, row block order. z holds r on entry and y on exit.
template <class T>
__global__ void __launch_bounds__(256) k_trsv_fwd(const T* __restrict__ M, int ld, const T* __restrict__ Linv, int nb,
                                                  double* z, unsigned* flags, unsigned epoch, int* err) {
  __shared__ double part[4][kNB];
  __shared__ double ys[kSolveBatch][kNB];
  __shared__ double rhs[kNB];
  __shared__ int s_run;
  const int t = threadIdx.x, r = t & (kNB - 1), g = t >> 6;
  for (int i = blockIdx.x; i < nb; i += gridDim.x) {
    // this thread's 16 entries of Linv_ii and of L_{i,i-1} (the last dependency), loaded before any
    // wait: once block i-1 releases its flag, the remaining path has no global loads of L
    double li[16], lp[16];
    const T* Li = Linv + static_cast<int64_t>(i) * kNB * kNB;
#pragma unroll
    for (int u = 0; u < 16; ++u) li[u] = static_cast<double>(Li[(g * 16 + u) * kNB + r]);
    if (i > 0) {
      const T* Lp = M + static_cast<int64_t>((i - 1) * kNB) * ld + i * kNB + r;
#pragma unroll
      for (int u = 0; u < 16; ++u) lp[u] = static_cast<double>(Lp[static_cast<int64_t>(g * 16 + u) * ld]);
    }
    double acc = 0.0;
    bool bad = false;
    // blocks 0 .. i-2 in runs of released ones (one flag check per run, not per block)
    for (int done = 0; done < i - 1;) {
      if (t < 32) {
        const int run = released_run(flags, done, 1, min(kSolveBatch, i - 1 - done), epoch);
        if (t == 0) s_run = run;
      }
      __syncthreads();
      const int run = s_run;
      if (run == 0) {
        bad = true;
        break;
      }
      for (int idx = t; idx < run * kNB; idx += blockDim.x)
        ys[idx / kNB][idx % kNB] = __ldcg(z + (done + idx / kNB) * kNB + idx % kNB);
      __syncthreads();
#pragma unroll 2
      for (int b = 0; b < run; ++b) {
        const T* Lij = M + static_cast<int64_t>((done + b) * kNB) * ld + i * kNB + r;
#pragma unroll
        for (int u = 0; u < 16; ++u)
          acc += static_cast<double>(Lij[static_cast<int64_t>(g * 16 + u) * ld]) * ys[b][g * 16 + u];
      }
      __syncthreads();
      done += run;
    }
    if (i > 0 && !bad) {
      if (t < 32) {
        const int run = released_run(flags, i - 1, 1, 1, epoch);
        if (t == 0) s_run = run;
      }
      __syncthreads();
      if (s_run == 0) {
        bad = true;
      } else {
        if (t < kNB) ys[0][t] = __ldcg(z + (i - 1) * kNB + t);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 16; ++u) acc += lp[u] * ys[0][g * 16 + u];
      }
    }
    if (bad && t == 0) atomicExch(err, 1);
    part[g][r] = acc;
    __syncthreads();
    if (t < kNB) rhs[t] = z[i * kNB + t] - (part[0][t] + part[1][t] + part[2][t] + part[3][t]);
    __syncthreads();
    double y = 0.0;
#pragma unroll
    for (int u = 0; u < 16; ++u) y += li[u] * rhs[g * 16 + u];
    part[g][r] = y;
    __syncthreads();
    if (t < kNB) z[i * kNB + t] = part[0][t] + part[1][t] + part[2][t] + part[3][t];
    __threadfence();
    __syncthreads();
    if (t == 0) st_release(flags + i, epoch);
  }
}

// Backward: L^T x = y, reverse row block order. Warp w handles columns c = 8w..8w+7 of a block.
template <class T>
__global__ void __launch_bounds__(256) k_trsv_bwd(const T* __restrict__ M, int ld, const T* __restrict__ Linv, int nb,
                                                  double* z, unsigned* flags, unsigned epoch, int* err) {
  __shared__ double part[4][kNB];
  __shared__ double xs[kSolveBatch][kNB];
  __shared__ double rhs[kNB];
  __shared__ int s_run;
  // thread (c, g): column c of the row block's L entries, rows 16g .. 16g+15 of each tile, so a
  // thread's entries of a tile are 16 consecutive values (vector loads) and the four groups' partial
  // sums meet in shared memory once per block
  const int t = threadIdx.x, c = t & (kNB - 1), g = t >> 6;
  for (int q = blockIdx.x; q < nb; q += gridDim.x) {
    const int i = nb - 1 - q;
    // this thread's entries of Linv_ii and of L_{i+1,i} (the last dependency), loaded before any wait
    double li[16], lp[16];
    const T* Li = Linv + static_cast<int64_t>(i) * kNB * kNB + c * kNB + g * 16;
    load16(Li, li);
    const T* colc = M + static_cast<int64_t>(i * kNB + c) * ld + g * 16;  // column i*64+c of L
    if (i + 1 < nb) load16(colc + (i + 1) * kNB, lp);
    double acc = 0.0;
    bool bad = false;
    // blocks nb-1 down to i+2 in runs of released ones
    const int deps = nb - i - 2;
    for (int done = 0; done < deps;) {
      const int j0 = nb - 1 - done;
      if (t < 32) {
        const int run = released_run(flags, j0, -1, min(kSolveBatch, deps - done), epoch);
        if (t == 0) s_run = run;
      }
      __syncthreads();
      const int run = s_run;
      if (run == 0) {
        bad = true;
        break;
      }
      for (int idx = t; idx < run * kNB; idx += blockDim.x)
        xs[idx / kNB][idx % kNB] = __ldcg(z + (j0 - idx / kNB) * kNB + idx % kNB);
      __syncthreads();
      // acc_c += sum_r L[j*64 + r][i*64 + c] * x_j[r], this thread's 16 rows r
#pragma unroll 2
      for (int b = 0; b < run; ++b) {
        double l[16];
        load16(colc + (j0 - b) * kNB, l);
#pragma unroll
        for (int u = 0; u < 16; ++u) acc += l[u] * xs[b][g * 16 + u];
      }
      __syncthreads();
      done += run;
    }
    if (i + 1 < nb && !bad) {
      if (t < 32) {
        const int run = released_run(flags, i + 1, 1, 1, epoch);
        if (t == 0) s_run = run;
      }
      __syncthreads();
      if (s_run == 0) {
        bad = true;
      } else {
        if (t < kNB) xs[0][t] = __ldcg(z + (i + 1) * kNB + t);
        __syncthreads();
#pragma unroll
        for (int u = 0; u < 16; ++u) acc += lp[u] * xs[0][g * 16 + u];
      }
    }
    if (bad && t == 0) atomicExch(err, 1);
    part[g][c] = acc;
    __syncthreads();
    if (t < kNB) rhs[t] = z[i * kNB + t] - (part[0][t] + part[1][t] + part[2][t] + part[3][t]);
    __syncthreads();
    // x_c = sum_r Linv[r][c] rhs[r] = sum_r Li[c * 64 + r] rhs[r]
    double y = 0.0;
#pragma unroll
    for (int u = 0; u < 16; ++u) y += li[u] * rhs[g * 16 + u];
    part[g][c] = y;
    __syncthreads();
    if (t < kNB) z[i * kNB + t] = part[0][t] + part[1][t] + part[2][t] + part[3][t];
    __threadfence();
    __syncthreads();
    if (t == 0) st_release(flags + i, epoch);
  }
}

// Co-resident blocks of the cooperative solves, per device (queried once per device).
int dataflow_grid(int nb) {
  static int max_blocks[kMaxDevices] = {};
  int dev = 0;
  SOV_CUDA(cudaGetDevice(&dev));
  if (dev >= kMaxDevices) throw std::runtime_error("dense solve: device index beyond the supported 64");
  once_per_device((const void*)&max_blocks, [&] {
    int sms = 0, per_sm = 0;
    SOV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SOV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_trsv_fwd<double>, 256, 0));
    max_blocks[dev] = std::max(1, sms * std::max(1, per_sm));
  });
  std::lock_guard<std::mutex> g(once_mutex());  // the write above happened under this lock
  return std::min(nb, max_blocks[dev]);
}

template <class T>
void dense_solve(const DenseSystem<T>& s, double* z, unsigned& epoch, int* err, cudaStream_t st, int* launches) {
  const int grid = dataflow_grid(s.nb);
  const T* M = s.M;
  const T* Linv = s.Linv;
  int ld = s.mp, nb = s.nb;
  unsigned e1 = ++epoch;
  void* args1[] = {(void*)&M, (void*)&ld, (void*)&Linv, (void*)&nb, (void*)&z, (void*)&s.flags, (void*)&e1, (void*)&err};
  SOV_CUDA(cudaLaunchCooperativeKernel((const void*)k_trsv_fwd<T>, dim3(grid), dim3(256), args1, 0, st));
  unsigned e2 = ++epoch;
  void* args2[] = {(void*)&M, (void*)&ld, (void*)&Linv, (void*)&nb, (void*)&z, (void*)&s.flags, (void*)&e2, (void*)&err};
  SOV_CUDA(cudaLaunchCooperativeKernel((const void*)k_trsv_bwd<T>, dim3(grid), dim3(256), args2, 0, st));
  if (launches) *launches += 2;
}

// explicit instantiations
template void launch_assemble<double>(const AssemblyDev&, const double*, const double*, const double*,
                                     const uint8_t*, int, double, double*, double*, int, int, cudaStream_t);
template void launch_assemble<float>(const AssemblyDev&, const double*, const double*, const double*,
                                    const uint8_t*, int, double, float*, double*, int, int, cudaStream_t);
template void launch_dense_clear<double>(double*, int, int, cudaStream_t);
template void launch_dense_clear<float>(float*, int, int, cudaStream_t);
template void dense_potrf_block<double>(const DenseSystem<double>&, int, cudaStream_t);
template void dense_potrf_block<float>(const DenseSystem<float>&, int, cudaStream_t);
template void dense_cholesky<double>(const DenseSystem<double>&, cudaStream_t, int*);
template void dense_cholesky<float>(const DenseSystem<float>&, cudaStream_t, int*);
template void dense_solve<double>(const DenseSystem<double>&, double*, unsigned&, int*, cudaStream_t, int*);
template void dense_solve<float>(const DenseSystem<float>&, double*, unsigned&, int*, cudaStream_t, int*);

}  // namespace sov
