// sparse_gpu.cu -- numeric sparse L D L' and its solves on the GPU (see sparse_gpu.cuh).
#include "sparse_gpu.cuh"

#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <stdexcept>

#include "common.cuh"

namespace cg = cooperative_groups;

namespace sov {
namespace {

constexpr int kSparseThreads = 256;

__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Per level: the pivots of its columns (one thread each), then its rank-1 updates, one warp per
// destination: lane l sums the destination's terms l, l + 32, ... and the warp adds the 32 partial
// sums in a fixed tree (deterministic).
__global__ void __launch_bounds__(kSparseThreads) k_sparse_factor(SparseDev s) {
  cg::grid_group g = cg::this_grid();
  const int rank = static_cast<int>(g.thread_rank()), size = static_cast<int>(g.size());
  const int lane = threadIdx.x & 31, warp = rank >> 5, warps = size >> 5;
  int drops = 0, bad = 0;
  for (int h = 0; h < s.levels; ++h) {
    for (int q = s.lvl_ptr[h] + rank; q < s.lvl_ptr[h + 1]; q += size) {
      const int k = s.lvl_col[q];
      const double p = s.V[k];
      const double sg = s.sign ? static_cast<double>(s.sign[k]) : 1.0;
      const bool finite = fabs(p) <= 1.7976931348623157e308;
      const bool drop = !(finite && sg * p > s.drop_tol * fabs(s.diag[k]));
      bad |= !finite;
      drops += drop;
      s.inv_d[k] = 1.0 / (drop ? sg * 1e128 : p);
    }
    g.sync();
    for (int r = s.run_lvl[h] + warp; r < s.run_lvl[h + 1]; r += warps) {
      double acc = 0.0;
      for (int u = s.run_ptr[r] + lane; u < s.run_ptr[r + 1]; u += 32)
        acc += s.V[s.m + s.up_a[u]] * s.V[s.m + s.up_b[u]] * s.inv_d[s.up_col[u]];
      acc = warp_total(acc);
      if (lane == 0) s.V[s.run_dst[r]] -= acc;
    }
    g.sync();
  }
  if (drops) atomicAdd(s.drop_count, drops);
  if (bad) atomicExch(s.fail, 1);
}

// L D L' x = z: forward y_k = z_k - sum_j L~_kj (1/D_j) y_j (row k of L, descendants: earlier
// levels), backward x_k = (1/D_k) (y_k - sum_i L~_ik x_i) (column k, ancestors: later levels);
// one warp per column, partial sums added in a fixed tree
__global__ void __launch_bounds__(kSparseThreads) k_sparse_solve(SparseDev s, double* z, const int* run) {
  if (run && !*run) return;  // written by an earlier launch: every block takes the same exit
  cg::grid_group g = cg::this_grid();
  const int rank = static_cast<int>(g.thread_rank()), size = static_cast<int>(g.size());
  const int lane = threadIdx.x & 31, warp = rank >> 5, warps = size >> 5;
  for (int k = rank; k < s.m; k += size) s.work[k] = z[s.perm[k]];
  g.sync();
  for (int h = 0; h < s.levels; ++h) {
    for (int q = s.lvl_ptr[h] + warp; q < s.lvl_ptr[h + 1]; q += warps) {
      const int k = s.lvl_col[q];
      double acc = 0.0;
      for (int t = s.row_ptr[k] + lane; t < s.row_ptr[k + 1]; t += 32)
        acc += s.V[s.m + s.row_pos[t]] * s.inv_d[s.row_col[t]] * s.work[s.row_col[t]];
      acc = warp_total(acc);
      if (lane == 0) s.work[k] -= acc;
    }
    g.sync();
  }
  for (int h = s.levels - 1; h >= 0; --h) {
    for (int q = s.lvl_ptr[h] + warp; q < s.lvl_ptr[h + 1]; q += warps) {
      const int k = s.lvl_col[q];
      double acc = 0.0;
      for (int p = s.lp[k] + lane; p < s.lp[k + 1]; p += 32) acc += s.V[s.m + p] * s.work[s.li[p]];
      acc = warp_total(acc);
      if (lane == 0) s.work[k] = (s.work[k] - acc) * s.inv_d[k];
    }
    g.sync();
  }
  for (int k = rank; k < s.m; k += size) z[s.perm[k]] = s.work[k];
}

template <class T>
T* put(std::vector<void*>& bufs, const std::vector<T>& h, cudaStream_t st) {
  T* p = nullptr;
  SOV_CUDA(cudaMalloc(&p, sizeof(T) * std::max<size_t>(1, h.size())));
  bufs.push_back(p);
  if (!h.empty()) SOV_CUDA(cudaMemcpyAsync(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice, st));
  return p;
}

}  // namespace

void SparseFactor::upload(const SparseSymbolic& s, int* drop_count, int* fail, double drop_tol, cudaStream_t st,
                          const std::vector<int8_t>* sign) {
  release();
  const int m = s.m, levels = s.levels();
  nnz_l_ = s.nnz_l;
  // updates grouped by (level, destination), schedule order kept within a group: two stable
  // counting sorts (by destination, then by level), linear in the number of updates
  const size_t n_up = s.pairs.size() / 4;
  const int n_dst = m + static_cast<int>(s.li.size());
  std::vector<int> level_of(n_up);
  for (int h = 0; h < levels; ++h)
    for (int u = s.pair_ptr[h]; u < s.pair_ptr[h + 1]; ++u) level_of[u] = h;
  std::vector<int> by_dst(n_up), order(n_up);
  {
    std::vector<size_t> cnt(n_dst + 1, 0);
    for (size_t u = 0; u < n_up; ++u) cnt[s.pairs[4 * u + 3] + 1]++;
    for (int d = 0; d < n_dst; ++d) cnt[d + 1] += cnt[d];
    for (size_t u = 0; u < n_up; ++u) by_dst[cnt[s.pairs[4 * u + 3]]++] = static_cast<int>(u);
    std::vector<size_t> lc(levels + 1, 0);
    for (size_t u = 0; u < n_up; ++u) lc[level_of[u] + 1]++;
    for (int h = 0; h < levels; ++h) lc[h + 1] += lc[h];
    for (size_t q = 0; q < n_up; ++q) {
      const int u = by_dst[q];
      order[lc[level_of[u]]++] = u;
    }
  }
  std::vector<int> run_lvl(levels + 1, 0), run_ptr(1, 0), run_dst, up_col(n_up), up_a(n_up), up_b(n_up);
  run_dst.reserve(n_up);
  run_ptr.reserve(n_up + 1);
  for (size_t q = 0; q < n_up; ++q) {
    const int u = order[q];
    const bool new_run = q == 0 || level_of[u] != level_of[order[q - 1]] || s.pairs[4 * u + 3] != run_dst.back();
    if (new_run) {
      if (q > 0) run_ptr.push_back(static_cast<int>(q));
      run_dst.push_back(s.pairs[4 * u + 3]);
      run_lvl[level_of[u] + 1] = static_cast<int>(run_dst.size());
    }
    up_col[q] = s.pairs[4 * u];
    up_a[q] = s.pairs[4 * u + 1];
    up_b[q] = s.pairs[4 * u + 2];
  }
  if (n_up) run_ptr.push_back(static_cast<int>(n_up));
  for (int h = 0; h < levels; ++h) run_lvl[h + 1] = std::max(run_lvl[h + 1], run_lvl[h]);
  // rows of L for the forward solve
  std::vector<int> row_ptr(m + 1, 0), row_pos(s.li.size()), row_col(s.li.size());
  for (int i : s.li) row_ptr[i + 1]++;
  for (int i = 0; i < m; ++i) row_ptr[i + 1] += row_ptr[i];
  {
    std::vector<int> fill(row_ptr.begin(), row_ptr.end() - 1);
    for (int k = 0; k < m; ++k)
      for (int p = s.lp[k]; p < s.lp[k + 1]; ++p) {
        const int t = fill[s.li[p]]++;
        row_pos[t] = p;
        row_col[t] = k;
      }
  }
  d_.m = m;
  d_.levels = levels;
  std::vector<double> zeros;
  d_.V = put(bufs_, std::vector<double>(m + s.li.size(), 0.0), st);
  d_.diag = put(bufs_, std::vector<double>(m, 0.0), st);
  d_.inv_d = put(bufs_, std::vector<double>(m, 0.0), st);
  d_.work = put(bufs_, std::vector<double>(m, 0.0), st);
  d_.perm = put(bufs_, s.perm, st);
  d_.lp = put(bufs_, s.lp, st);
  d_.li = put(bufs_, s.li, st);
  d_.lvl_ptr = put(bufs_, s.lvl_ptr, st);
  d_.lvl_col = put(bufs_, s.lvl_col, st);
  d_.run_lvl = put(bufs_, run_lvl, st);
  d_.run_ptr = put(bufs_, run_ptr, st);
  d_.run_dst = put(bufs_, run_dst, st);
  d_.up_col = put(bufs_, up_col, st);
  d_.up_a = put(bufs_, up_a, st);
  d_.up_b = put(bufs_, up_b, st);
  d_.row_ptr = put(bufs_, row_ptr, st);
  d_.row_pos = put(bufs_, row_pos, st);
  d_.row_col = put(bufs_, row_col, st);
  d_.drop_count = drop_count;
  d_.fail = fail;
  d_.drop_tol = drop_tol;
  d_.sign = nullptr;
  std::vector<int8_t> sign_elim;
  if (sign) {
    sign_elim.resize(m);
    for (int k = 0; k < m; ++k) sign_elim[k] = (*sign)[s.perm[k]];
    d_.sign = put(bufs_, sign_elim, st);
  }
  SOV_CUDA(cudaStreamSynchronize(st));  // the host vectors above go out of scope
  int dev = 0, sms = 0, per_sm = 0;
  SOV_CUDA(cudaGetDevice(&dev));
  SOV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SOV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sparse_factor, kSparseThreads, 0));
  int per_sm2 = 0;
  SOV_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_sparse_solve, kSparseThreads, 0));
  // one CTA per SM: most levels hold few columns, and a grid barrier costs more with more CTAs
  grid_ = std::max(1, sms * std::min(1, std::min(per_sm, per_sm2)));
}

void SparseFactor::release() {
  for (void* p : bufs_) cudaFree(p);
  bufs_.clear();
  d_ = SparseDev{};
}

void SparseFactor::factor(cudaStream_t st, int* launches) {
  SparseDev d = d_;
  void* args[] = {&d};
  SOV_CUDA(cudaLaunchCooperativeKernel((const void*)k_sparse_factor, dim3(grid_), dim3(kSparseThreads), args, 0, st));
  if (launches) *launches += 1;
}

void SparseFactor::solve(double* z, cudaStream_t st, int* launches, const int* run) {
  SparseDev d = d_;
  void* args[] = {&d, &z, &run};
  SOV_CUDA(cudaLaunchCooperativeKernel((const void*)k_sparse_solve, dim3(grid_), dim3(kSparseThreads), args, 0, st));
  if (launches) *launches += 1;
}

}  // namespace sov
