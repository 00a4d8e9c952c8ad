// dense.cuh -- dense normal-matrix path: assembly, blocked Cholesky, dataflow triangular solves.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace sov {

constexpr int kNB = 64;             // tile / panel width of the blocked factorization
constexpr double kBigPivotD = 1e64; // a dropped pivot's L_jj (D_jj = 1e128, sparse_ldlt.cpp:170)
constexpr float kBigPivotF = 1e19f; // FP32 counterpart (D_jj = 1e38)

// Device view of one dense normal-equation system of order m, padded to mp (multiple of kNB).
template <class T>
struct DenseSystem {
  T* M;              // mp x mp column-major, lower triangle used; padding rows/cols = identity
  T* Linv;           // (mp/kNB) blocks of kNB x kNB: inverses of the diagonal blocks of L
  double* diag;      // m: diagonal of M + regularization before elimination (pivot-drop rule)
  int m, mp, nb;
  int* drop_count;   // dropped pivots (dependent rows)
  int* fail;         // non-finite pivot
  unsigned* flags;   // nb: dataflow flags for the factor's panels and the triangular solves
  unsigned* tickets; // 1: work-item counter of the factor's panel launches
  double drop_tol;   // pivot <= drop_tol * diag is a dependent row (1e-13 FP64, looser for FP32)
};

// M = A diag(d) A' + reg I via the gather map (one thread per target entry). The column
// weight d_k is computed on the fly from the iterate:
//   LP: d = max(x,1e-16)/max(s,1e-16)                  (interior_point.cpp:411-415)
//   QP: d = 1/(qdiag + h), h = free ? 0 : max(s,1e-16)/max(x,1e-16)  (qp_interior_point.cpp:449-456)
//   ones: d = 1 (the starting-point system: LP interior_point.cpp:490-491; QP H = I, the KKT factored
//   without the Hessian, qp_interior_point.cpp:2884 and :449-456)
//   theta: d = max(s,1e-16)/max(x,1e-16) of the given column (x-space QP: the slack's barrier weight)
enum WeightMode : int { kWeightLp = 0, kWeightQp = 1, kWeightOnes = 2, kWeightTheta = 3 };

struct AssemblyDev {
  const int64_t* target;
  const int* ptr;
  const int* col;
  const double* w;
  const int* diag_target;
  int ntargets;
};

template <class T>
void launch_assemble(const AssemblyDev& am, const double* x, const double* s, const double* qdiag,
                     const uint8_t* free_col, int mode, double reg, T* out, double* diag_out, int m,
                     int layout_ld, cudaStream_t st);  // layout_ld > 0 dense (leading dim), < 0 band (-m)

// Zero the lower triangle and put 1 on the padding diagonal.
template <class T>
void launch_dense_clear(T* M, int m, int mp, cudaStream_t st);

// Blocked right-looking Cholesky M = L L' in place. Pivots below 1e-13 * diag are replaced by
// kBigPivot (the reference's dependent-row rule, sparse_ldlt.cpp:165-173 with the threshold of
// interior_point.cpp:160); a non-finite pivot sets *fail.
template <class T>
void dense_cholesky(const DenseSystem<T>& s, cudaStream_t st, int* launches);

// One diagonal block of the blocked factorization (factor + inverse), stream-ordered.
template <class T>
void dense_potrf_block(const DenseSystem<T>& s, int kb, cudaStream_t st);

// FP32 factorization with the panel and trailing products as 3xTF32 tcgen05 MMAs (tc_chol.cu).
void dense_cholesky_tc(const DenseSystem<float>& s, int* err, cudaStream_t st, int* launches);

// In-place solve of L L' z = r for one FP64 right-hand side of length mp (padding entries 0).
template <class T>
void dense_solve(const DenseSystem<T>& s, double* z, unsigned& epoch, int* err, cudaStream_t st,
                 int* launches);

// Number of CTAs the dataflow solve may use (all co-resident).
int dataflow_grid(int nb);

}  // namespace sov
