// sparse.hpp -- host ordering and symbolic analysis for the sparse LDL' of the normal matrix.
//
// Approximate minimum-degree ordering of A A' on its quotient graph (Amestoy, Davis & Duff 1996:
// eliminated rows become elements, degrees are the paper's upper bound, rows denser than
// max(16, 10 sqrt(m)) are ordered last, an optional fill limit aborts the analysis), then the
// column patterns of L, the elimination tree and a level schedule for the GPU: columns of equal
// height in the tree have no ancestor relation, so a level's columns are finished together and
// their rank-1 updates applied together. The reference orders with its own minimum degree
// (solver/numerical/src/amd_ordering.cpp:12-130); the orders differ, the factorization does not
// depend on which fill-reducing order is used.
#pragma once

#include <cstdint>
#include <vector>

#include "stdform.hpp"

namespace sov {

// Fill-reducing order: approximate minimum degree, nested dissection, or (kAuto) minimum degree
// unless its elimination tree is deep and the dissection order's estimated GPU factor time is
// lower.
enum class SparseOrder { kAuto, kMinimumDegree, kNestedDissection };

struct SparseSymbolic {
  int m = 0;
  SparseOrder ordering = SparseOrder::kMinimumDegree;  // the order taken
  std::vector<int> perm, iperm;  // perm[k] = row eliminated k-th; iperm[row] = k
  std::vector<int> lp, li;       // L (permuted): column k's strict-lower rows li[lp[k]..lp[k+1]), ascending
  std::vector<int> parent;       // elimination tree (permuted), -1 at roots
  std::vector<int> lvl_ptr, lvl_col;  // columns grouped by height in the tree (leaves first)
  // rank-1 updates of each level: (column k, position of l_ak, position of l_bk, destination);
  // destination < m is the diagonal slot of a row, else m + position in L
  std::vector<int> pair_ptr;     // per level
  std::vector<int> pairs;        // 4 ints per update
  // assembly of A diag(d) A' into the [D | L] storage: targets with their contributions
  std::vector<int> asm_target, asm_ptr, asm_col;
  std::vector<double> asm_w;
  long long nnz_l = 0;
  double flops = 0.0;            // sum over columns of colcount^2 (sparse_ldlt.cpp:230-238)
  int levels() const { return static_cast<int>(lvl_ptr.size()) - 1; }
};

// rank-1 update terms the schedule may hold (16 bytes each on the device)
constexpr double kMaxUpdates = 2e8;

// Returns false when the predicted fill exceeds fill_limit entries (0 = no limit) or the update
// schedule would exceed kMaxUpdates terms.
bool sparse_analyze(const StdForm& f, std::size_t fill_limit, SparseSymbolic& out,
                    SparseOrder order = SparseOrder::kAuto);

// The same analysis for any symmetric pattern (adjacency lists without the diagonal, both
// directions), without an assembly map: the caller places its values with sparse_slot.
bool sparse_analyze_graph(const std::vector<std::vector<int>>& adj, std::size_t fill_limit, SparseSymbolic& out,
                          SparseOrder order = SparseOrder::kAuto);

// Index into the [D | L] value storage of entry (i, j) of the original ordering (-1 if it is not
// in the pattern of L).
int sparse_slot(const SparseSymbolic& s, int i, int j);

// The GPU work schedule of a symbolic factor. Work items -- a destination's run of rank-1 terms
// (factor), a row of L (forward solve), a column of L (backward solve) -- are cut into pieces of
// at most kSparsePiece terms, one warp each, so that one long item (a dense row's diagonal collects
// a term from nearly every column) spreads over many warps. A piece with slot < 0 applies its sum
// to its target directly; otherwise the sum goes to partial[slot], and the level's combine entry
// {target, first slot, slots} adds the item's partial sums in order after one more grid barrier.
constexpr int kSparsePiece = 1024;

struct SparsePiece {
  int first, end, target, slot;  // same layout as the device's int4
};
struct SparseCombine {
  int target, first, count, pad;
};
// Within a level, pieces of at most kSparseShort terms come first, one thread each (most items of
// a sparse factor are a few terms long: a warp per item would leave most lanes idle); the longer
// pieces follow from warp_lvl[h] on, one warp each.
constexpr int kSparseShort = 16;
struct SparsePieces {
  std::vector<SparsePiece> piece;
  std::vector<SparseCombine> comb;
  std::vector<int> piece_lvl{0}, comb_lvl{0};  // per level
  std::vector<int> warp_lvl;                   // per level: first piece taken by a warp
  std::vector<SparsePiece> pending_long;       // while a level is built
};
struct SparseSchedule {
  // updates in (level, destination) order
  std::vector<int> up_col, up_a, up_b;  // pivot column, positions of l_ak and l_bk
  SparsePieces factor;                  // over the update range; target = index into [D | L]
  std::vector<int> row_pos, row_col;    // entries of L by row: positions in L, columns
  SparsePieces forward;                 // over row_pos / row_col; target = row k
  SparsePieces backward;                // over li; target = column k (every column has a piece)
  int factor_slots = 0, solve_slots = 0;
  // with a dense tail (tail > 0): the last `tail` columns are left out of the level schedule --
  // their pivots, their update terms and their columns in the backward solve -- for a dense
  // factorization and dense solves of that block; `levels` levels remain (pivot_ptr/pivot_col:
  // their columns), and the forward solve has one more level, the tail rows' sums over the
  // columns before the tail
  int tail = 0, levels = 0;
  std::vector<int> pivot_ptr, pivot_col;
};

// piece: the longest piece (items beyond it are cut); a schedule walked by one thread per piece
// takes short pieces
SparseSchedule sparse_schedule(const SparseSymbolic& s, int tail = 0, int piece = kSparsePiece);

// The trailing columns of L whose pattern is every later row (a dense trailing block: the root
// clique of the elimination tree). Their L entries are stored column by column, rows ascending,
// so the block is a column-packed lower triangle inside [D | L].
int sparse_dense_tail(const SparseSymbolic& s);

// The trailing block worth factoring densely: the T (at least the dense tail) minimizing
// sparse_cost * (rank-1 terms left to the level schedule) + (T^3 / 6 dense multiply-adds), the
// explicit zeros of a nearly dense block included. sparse_cost: a scheduled term's cost in dense
// multiply-adds. 0 when no block of at least min_block columns pays.
int sparse_dense_block(const SparseSymbolic& s, double sparse_cost, int min_block);

// The rows of a CSR pattern (ptr, rows + 1 entries) as pieces of one level: target = row; the
// combine entries hold the rows that were cut, slots numbered from 0.
SparsePieces row_pieces(const std::vector<int>& ptr, int* slots);

}  // namespace sov
