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
// piece: lane l sums the piece's terms l, l + 32, ... and the warp adds the 32 partial sums in a
// fixed tree; a run cut into pieces is finished by its combine step (deterministic either way).
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
    for (int q = s.fpiece_lvl[h] + rank; q < s.fwarp_lvl[h]; q += size) {  // short pieces: a thread each
      const int4 pc = s.fpiece[q];
      double acc = 0.0;
      for (int u = pc.x; u < pc.y; ++u) acc += s.V[s.m + s.up_a[u]] * s.V[s.m + s.up_b[u]] * s.inv_d[s.up_col[u]];
      if (pc.w < 0) s.V[pc.z] -= acc;
      else s.partial[pc.w] = acc;
    }
    for (int q = s.fwarp_lvl[h] + warp; q < s.fpiece_lvl[h + 1]; q += warps) {
      const int4 pc = s.fpiece[q];
      double acc = 0.0;
      for (int u = pc.x + lane; u < pc.y; u += 32)
        acc += s.V[s.m + s.up_a[u]] * s.V[s.m + s.up_b[u]] * s.inv_d[s.up_col[u]];
      acc = warp_total(acc);
      if (lane == 0) {
        if (pc.w < 0) s.V[pc.z] -= acc;
        else s.partial[pc.w] = acc;
      }
    }
    if (s.fcomb_lvl[h + 1] > s.fcomb_lvl[h]) {  // uniform: every thread reads the same bounds
      g.sync();
      for (int c = s.fcomb_lvl[h] + rank; c < s.fcomb_lvl[h + 1]; c += size) {
        const int4 cb = s.fcomb[c];
        double t = 0.0;
        for (int k = 0; k < cb.z; ++k) t += s.partial[cb.y + k];
        s.V[cb.x] -= t;
      }
    }
    g.sync();
  }
  if (drops) atomicAdd(s.drop_count, drops);
  if (bad) atomicExch(s.fail, 1);
}

// L D L' x = z: forward y_k = z_k - sum_j L~_kj (1/D_j) y_j (row k of L, descendants: earlier
// levels), backward x_k = (1/D_k) (y_k - sum_i L~_ik x_i) (column k, ancestors: later levels);
// one warp per piece, partial sums added in a fixed tree, long rows and columns through their
// combine steps
__global__ void __launch_bounds__(kSparseThreads) k_sparse_solve(SparseDev s, double* z, const int* run) {
  if (run && !*run) return;  // written by an earlier launch: every block takes the same exit
  cg::grid_group g = cg::this_grid();
  const int rank = static_cast<int>(g.thread_rank()), size = static_cast<int>(g.size());
  const int lane = threadIdx.x & 31, warp = rank >> 5, warps = size >> 5;
  for (int k = rank; k < s.m; k += size) s.work[k] = z[s.perm[k]];
  g.sync();
  for (int h = 0; h < s.levels; ++h) {
    for (int q = s.lpiece_lvl[h] + rank; q < s.lwarp_lvl[h]; q += size) {
      const int4 pc = s.lpiece[q];
      double acc = 0.0;
      for (int t = pc.x; t < pc.y; ++t) acc += s.V[s.m + s.row_pos[t]] * s.inv_d[s.row_col[t]] * s.work[s.row_col[t]];
      if (pc.w < 0) s.work[pc.z] -= acc;
      else s.partial[pc.w] = acc;
    }
    for (int q = s.lwarp_lvl[h] + warp; q < s.lpiece_lvl[h + 1]; q += warps) {
      const int4 pc = s.lpiece[q];
      double acc = 0.0;
      for (int t = pc.x + lane; t < pc.y; t += 32)
        acc += s.V[s.m + s.row_pos[t]] * s.inv_d[s.row_col[t]] * s.work[s.row_col[t]];
      acc = warp_total(acc);
      if (lane == 0) {
        if (pc.w < 0) s.work[pc.z] -= acc;
        else s.partial[pc.w] = acc;
      }
    }
    if (s.lcomb_lvl[h + 1] > s.lcomb_lvl[h]) {
      g.sync();
      for (int c = s.lcomb_lvl[h] + rank; c < s.lcomb_lvl[h + 1]; c += size) {
        const int4 cb = s.lcomb[c];
        double t = 0.0;
        for (int k = 0; k < cb.z; ++k) t += s.partial[cb.y + k];
        s.work[cb.x] -= t;
      }
    }
    g.sync();
  }
  for (int h = s.levels - 1; h >= 0; --h) {
    for (int q = s.upiece_lvl[h] + rank; q < s.uwarp_lvl[h]; q += size) {
      const int4 pc = s.upiece[q];
      double acc = 0.0;
      for (int p = pc.x; p < pc.y; ++p) acc += s.V[s.m + p] * s.work[s.li[p]];
      if (pc.w < 0) s.work[pc.z] = (s.work[pc.z] - acc) * s.inv_d[pc.z];
      else s.partial[pc.w] = acc;
    }
    for (int q = s.uwarp_lvl[h] + warp; q < s.upiece_lvl[h + 1]; q += warps) {
      const int4 pc = s.upiece[q];
      double acc = 0.0;
      for (int p = pc.x + lane; p < pc.y; p += 32) acc += s.V[s.m + p] * s.work[s.li[p]];
      acc = warp_total(acc);
      if (lane == 0) {
        if (pc.w < 0) s.work[pc.z] = (s.work[pc.z] - acc) * s.inv_d[pc.z];
        else s.partial[pc.w] = acc;
      }
    }
    if (s.ucomb_lvl[h + 1] > s.ucomb_lvl[h]) {
      g.sync();
      for (int c = s.ucomb_lvl[h] + rank; c < s.ucomb_lvl[h + 1]; c += size) {
        const int4 cb = s.ucomb[c];
        double t = 0.0;
        for (int k = 0; k < cb.z; ++k) t += s.partial[cb.y + k];
        s.work[cb.x] = (s.work[cb.x] - t) * s.inv_d[cb.x];
      }
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
  const SparseSchedule S = sparse_schedule(s);
  d_.m = m;
  d_.levels = levels;
  d_.V = put(bufs_, std::vector<double>(m + s.li.size(), 0.0), st);
  d_.diag = put(bufs_, std::vector<double>(m, 0.0), st);
  d_.inv_d = put(bufs_, std::vector<double>(m, 0.0), st);
  d_.work = put(bufs_, std::vector<double>(m, 0.0), st);
  d_.perm = put(bufs_, s.perm, st);
  d_.lp = put(bufs_, s.lp, st);
  d_.li = put(bufs_, s.li, st);
  d_.lvl_ptr = put(bufs_, s.lvl_ptr, st);
  d_.lvl_col = put(bufs_, s.lvl_col, st);
  static_assert(sizeof(SparsePiece) == sizeof(int4) && sizeof(SparseCombine) == sizeof(int4), "piece layout");
  auto put4 = [&](const auto& v) { return reinterpret_cast<const int4*>(put(bufs_, v, st)); };
  d_.fpiece = put4(S.factor.piece);
  d_.fpiece_lvl = put(bufs_, S.factor.piece_lvl, st);
  d_.fwarp_lvl = put(bufs_, S.factor.warp_lvl, st);
  d_.fcomb = put4(S.factor.comb);
  d_.fcomb_lvl = put(bufs_, S.factor.comb_lvl, st);
  d_.lpiece = put4(S.forward.piece);
  d_.lpiece_lvl = put(bufs_, S.forward.piece_lvl, st);
  d_.lwarp_lvl = put(bufs_, S.forward.warp_lvl, st);
  d_.lcomb = put4(S.forward.comb);
  d_.lcomb_lvl = put(bufs_, S.forward.comb_lvl, st);
  d_.upiece = put4(S.backward.piece);
  d_.upiece_lvl = put(bufs_, S.backward.piece_lvl, st);
  d_.uwarp_lvl = put(bufs_, S.backward.warp_lvl, st);
  d_.ucomb = put4(S.backward.comb);
  d_.ucomb_lvl = put(bufs_, S.backward.comb_lvl, st);
  d_.partial = put(bufs_, std::vector<double>(std::max(1, std::max(S.factor_slots, S.solve_slots)), 0.0), st);
  d_.up_col = put(bufs_, S.up_col, st);
  d_.up_a = put(bufs_, S.up_a, st);
  d_.up_b = put(bufs_, S.up_b, st);
  d_.row_pos = put(bufs_, S.row_pos, st);
  d_.row_col = put(bufs_, S.row_col, st);
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
