// kkt.cuh -- the quasi-definite KKT system of a QP whose Hessian couples variables, as a sparse
// L D L' on the GPU.
//
//   K = [ Q + X^-1 S + delta I    A'       ]      (n IPM columns, then m rows)
//       [ A                      -delta I  ]
//
// is the reference's QpKkt form (solver/qp/src/qp_interior_point.cpp:415-655): quasi-definite, so
// an L D L' exists for every symmetric ordering, with n positive and m negative pivots
// (:443-445); it is factored after the minimum-degree order of its pattern (the host analysis of
// sparse.hpp on the KKT graph) by the level-scheduled factor of sparse_gpu.cuh with signed pivots.
// delta starts at 1e-9 and grows x100 up to 1e-5 while a pivot comes out with the wrong sign or
// not finite, and never falls back below a value once needed (:459-466); every solve is refined
// against the system without delta, up to three steps, each kept only while it halves the
// residual's max-norm (:473-506, :612-633) -- decided on the device, no host round trip. Newton step: K [dx; -dy] = [r1; rp] with r1 = -rd + X^-1 rxs (free columns:
// -rd), the same step as the normal equations A H^-1 A' dy = rp - A H^-1 r1, dx = H^-1 (r1 + A'dy)
// without forming H^-1.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "sparse_gpu.cuh"
#include "stdform.hpp"

namespace sov {

struct KktDev {
  int n, m;
  const int *q_ptr, *q_idx;  // Q over the IPM columns, CSC, both triangles (diagonal included)
  const double* q_val;
  const double* qdiag;
  const int *col_ptr, *row_idx, *row_ptr, *col_idx;
  const double *cval, *rval;
  const uint8_t* free_col;
  const int* q_slot;      // per Q entry: its slot in [D | L] (strict lower triangle), else -1
  const int* a_slot;      // per A entry (CSC order): slot of (n + row, col)
  const int* xdiag_slot;  // n
  const int* ydiag_slot;  // m
  double* V;              // the factor's value storage
  double* diag;           // the assembled diagonal in elimination order (pivot reference)
  const int4* row_piece;  // the rows of A as warp-sized pieces (row_pieces in sparse.hpp)
  int row_pieces;
  const int4* row_comb;   // rows cut into pieces: {row, first slot, slots}
  int row_combs;
  double* row_partial;
};

class KktSystem {
 public:
  // Pattern, ordering, symbolic factor and value maps on the host; device copies on `st`.
  void build(const StdForm& f, const int* q_ptr_dev, const int* q_idx_dev, const double* q_val_dev,
             const double* qdiag_dev, const int* col_ptr_dev, const int* row_idx_dev, const double* cval_dev,
             const int* row_ptr_dev, const int* col_idx_dev, const double* rval_dev, const uint8_t* free_dev,
             int* drop_count, int* fail, cudaStream_t st);
  // Assemble with H = Q + X^-1 S (start: H = I) and factor, raising delta until every pivot has
  // its sign; returns false when even delta = 1e-5 fails.
  bool assemble_and_factor(bool start, const double* x, const double* s, cudaStream_t st, int* launches);
  // K [u; v] = [r1; rp]: dx = u (into r1_dx, in place), dy = -v (into dy), refined against the
  // system last assembled.
  void solve_newton(double* r1_dx, const double* rp, double* dy, cudaStream_t st, int* launches);
  // (A H^-1 A' + delta) z = rhs with the factored system (the normal-equation solve the starting
  // points use): K [u; v] = [0; rhs], z = -v; in place.
  void solve_normal(double* z, cudaStream_t st, int* launches);
  int order() const { return n_ + m_; }
  int factorizations() const { return factorizations_; }
  long long nnz_l() const { return sym_.nnz_l; }
  double flops() const { return sym_.flops; }
  const char* ordering() const {
    return sym_.ordering == SparseOrder::kNestedDissection ? "nested-dissection" : "minimum-degree";
  }
  int levels() const { return sym_.levels(); }
  double delta() const { return delta_; }
  ~KktSystem();

 private:
  static constexpr double kDeltaMin = 1e-9;  // kKktRegularization (qp_interior_point.cpp:389)
  static constexpr double kDeltaMax = 1e-5;  // kKktRegularizationMax (:390)
  void solve_refined(const double* top, const double* bottom, double* dx, double* dy, cudaStream_t st,
                     int* launches);
  void residual(const double* w, const double* c, double* res, unsigned long long* norm, const int* run,
                cudaStream_t st);
  int n_ = 0, m_ = 0;
  long long nq_ = 0, na_ = 0;
  double delta_ = kDeltaMin;
  bool start_ = false;
  const double* x_ = nullptr;  // the iterate the system was assembled at
  const double* s_ = nullptr;
  int factorizations_ = 0;
  int flags_h_[2] = {0, 0};
  SparseSymbolic sym_;
  SparseFactor factor_;
  KktDev d_{};
  int* fail_ = nullptr;
  int* drops_ = nullptr;
  std::vector<void*> bufs_;
  double *rhs_ = nullptr, *sol_ = nullptr, *res_ = nullptr, *cor_ = nullptr, *res2_ = nullptr;
  void* refine_ = nullptr;  // device refinement record
};

}  // namespace sov
