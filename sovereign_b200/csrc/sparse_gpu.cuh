// sparse_gpu.cuh -- numeric sparse L D L' of the normal matrix on the GPU, on the host's symbolic
// analysis (sparse.hpp: minimum-degree order, column patterns, elimination tree, level schedule).
//
// Storage V = [D | L~] in the elimination order: D_k at V[k], the strict-lower entries of column k
// (rows li[lp[k]..lp[k+1])) at V[m + p], kept unscaled (L~ = L D), so an update is
// a_ab -= L~_ak L~_bk / D_k. Columns of one level of the elimination tree have no ancestor relation:
// a level's pivots are taken together, then its rank-1 updates are applied, grouped per destination
// (each destination's contributions summed by one warp in a fixed order: deterministic). One
// cooperative launch per factorization and per solve, a grid barrier between levels.
// Pivot rule of the reference's sparse LDL' (sparse_ldlt.cpp:165-173): a pivot at most
// drop_tol * |assembled diagonal| (or not finite) marks a dependent row, D = 1e128; with a sign
// per pivot (quasi-definite systems) the test is sign * pivot, and a dropped pivot keeps its sign.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "sparse.hpp"

namespace sov {

struct SparseDev {
  int m, levels;
  double* V;            // m + nnz(L)
  double* diag;         // m: assembled diagonal (elimination order), the pivot reference
  double* inv_d;        // m
  double* work;         // m: permuted right-hand side / solution
  const int* perm;      // perm[k] = original row of the k-th pivot
  const int* lp;        // m + 1
  const int* li;        // nnz(L)
  const int* lvl_ptr;   // levels + 1
  const int* lvl_col;   // m
  // the work pieces and combine steps of sparse_schedule (sparse.hpp), per level
  const int4* fpiece;   // factor pieces (first, end: update range; target: index into V)
  const int* fpiece_lvl;  // levels + 1
  const int* fwarp_lvl;   // levels: first piece of the level taken by a warp (earlier: a thread)
  const int4* fcomb;    // factor combines {target, first slot, slots, 0}
  const int* fcomb_lvl;   // levels + 1
  const int4* lpiece;   // forward pieces (first, end: range of row_pos / row_col; target: row k)
  const int* lpiece_lvl;
  const int* lwarp_lvl;
  const int4* lcomb;
  const int* lcomb_lvl;
  const int4* upiece;   // backward pieces (first, end: range of li; target: column k)
  const int* upiece_lvl;
  const int* uwarp_lvl;
  const int4* ucomb;
  const int* ucomb_lvl;
  double* partial;      // piece sums awaiting their combine step
  const int* up_col;    // updates: pivot column k
  const int* up_a;      // updates: position of l_ak
  const int* up_b;      // updates: position of l_bk
  const int* row_pos;   // entries of L by row (forward solve): positions in L
  const int* row_col;   // their columns
  int* drop_count;
  int* fail;
  double drop_tol;
  const int8_t* sign;   // m (elimination order): the expected sign of each pivot, or null (all +1);
                        // a quasi-definite KKT matrix has +1 on its primal block, -1 on its dual
};

// Device copies of the schedule; owns its buffers.
class SparseFactor {
 public:
  // sign (optional, original ordering): the expected sign of each pivot (default all +1)
  void upload(const SparseSymbolic& s, int* drop_count, int* fail, double drop_tol, cudaStream_t st,
              const std::vector<int8_t>* sign = nullptr);
  void release();
  ~SparseFactor() { release(); }
  const SparseDev& dev() const { return d_; }
  double* values() const { return d_.V; }
  double* assembled_diag() const { return d_.diag; }
  long long nnz_l() const { return nnz_l_; }
  void factor(cudaStream_t st, int* launches);
  // z in the original row order, in place; run (optional, device): the solve is skipped when *run == 0
  void solve(double* z, cudaStream_t st, int* launches, const int* run = nullptr);

 private:
  SparseDev d_{};
  std::vector<void*> bufs_;
  long long nnz_l_ = 0;
  int grid_ = 1;
};

}  // namespace sov
