// kkt.cu -- quasi-definite KKT system of a coupled-Hessian QP, sparse L D L' on the GPU (kkt.cuh).
#include "kkt.cuh"

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>

#include "common.cuh"

namespace sov {
namespace {

constexpr int kKktThreads = 256;
constexpr int kKktRefineSteps = 3;  // kRefinementSteps (qp_interior_point.cpp:391)

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

int blocks_for(long long work) {
  return static_cast<int>(std::max(1LL, std::min(4096LL, (work + kKktThreads - 1) / kKktThreads)));
}

__device__ __forceinline__ double barrier_weight(const KktDev& d, const double* x, const double* s, int j) {
  return d.free_col[j] ? 0.0 : fmax(s[j], 1e-16) / fmax(x[j], 1e-16);
}

// V (zeroed) <- K; start: H = I and no Q terms. diag <- |K_kk| in elimination order.
__global__ void k_kkt_assemble(KktDev d, const double* x, const double* s, int start, double delta) {
  const int n = d.n, m = d.m;
  const int nq = d.q_ptr[n], na = d.col_ptr[n];
  const long long work = max(max(n, m), max(nq, na));
  for (long long t = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; t < work;
       t += static_cast<long long>(gridDim.x) * blockDim.x) {
    if (t < n) {
      const int j = static_cast<int>(t);
      const double v = (start ? 1.0 : d.qdiag[j] + barrier_weight(d, x, s, j)) + delta;
      d.V[d.xdiag_slot[j]] = v;
      d.diag[d.xdiag_slot[j]] = fabs(v);
    }
    if (t < m) {
      const int i = static_cast<int>(t);
      d.V[d.ydiag_slot[i]] = -delta;
      d.diag[d.ydiag_slot[i]] = delta;
    }
    if (!start && t < nq && d.q_slot[t] >= 0) atomicAdd(d.V + d.q_slot[t], d.q_val[t]);
    if (t < na) d.V[d.a_slot[t]] = d.cval[t];
  }
}

// Refinement bookkeeping of one solve (qp_interior_point.cpp:473-506): err[r] = |residual|_inf at
// the start of step r (bits of a non-negative double, so atomicMax orders them), next[r] = that of
// the candidate of step r; run[r] = step r executes, acc[r] = its candidate was kept. Each launch
// only reads slots that earlier launches wrote.
struct KktRefine {
  unsigned long long err[kKktRefineSteps + 1];
  unsigned long long next[kKktRefineSteps];
  int run[kKktRefineSteps];
  int acc[kKktRefineSteps];
};

__device__ __forceinline__ double bits_to(unsigned long long b) { return __longlong_as_double(static_cast<long long>(b)); }

__device__ __forceinline__ void record_norm(unsigned long long* norm, double local, bool nan) {
  local = warp_max(local);
  // a NaN residual records the quiet-NaN bits, above every finite and infinite norm: neither
  // "err > 0" nor "next < err / 2" holds for it
  nan = __any_sync(0xffffffffu, nan);
  const unsigned long long bits =
      nan ? 0x7ff8000000000000ULL : static_cast<unsigned long long>(__double_as_longlong(local));
  if ((threadIdx.x & 31) == 0) atomicMax(norm, bits);
}

// Residual res = rhs - K0 (w + c) (c may be null) with K0 = [Q + X^-1 S, A'; A, 0], the system
// without delta (start: [I, A'; A, 0]); |res|_inf into *norm. Skipped when run is given and
// *run == 0. Column rows (the first n) one thread each; the rows of A as pieces, a warp each (a
// dense row is cut into pieces, finished by k_kkt_residual_combine).
struct ResidualArgs {
  const double *x, *s;
  int start;
  const double *rhs, *w, *c;
  double* res;
  unsigned long long* norm;
  const int* run;
};

__global__ void k_kkt_residual(KktDev d, ResidualArgs a) {
  if (a.run && !*a.run) return;
  const int n = d.n;
  auto at = [&](int i) { return a.c ? a.w[i] + a.c[i] : a.w[i]; };
  double local = 0.0;
  bool nan = false;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  for (int j = tid; j < n; j += nthreads) {
    double acc = 0.0;
    if (a.start) {
      acc = at(j);
    } else {
      for (int k = d.q_ptr[j]; k < d.q_ptr[j + 1]; ++k) acc += d.q_val[k] * at(d.q_idx[k]);
      acc += barrier_weight(d, a.x, a.s, j) * at(j);
    }
    for (int p = d.col_ptr[j]; p < d.col_ptr[j + 1]; ++p) acc += d.cval[p] * at(n + d.row_idx[p]);
    const double e = a.rhs[j] - acc;
    a.res[j] = e;
    local = fmax(local, fabs(e));
    nan |= e != e;
  }
  const int lane = threadIdx.x & 31, warp = tid >> 5, warps = nthreads >> 5;
  for (int q = warp; q < d.row_pieces; q += warps) {
    const int4 pc = d.row_piece[q];
    double acc = 0.0;
    for (int p = pc.x + lane; p < pc.y; p += 32) acc += d.rval[p] * at(d.col_idx[p]);
    acc = warp_total(acc);
    if (pc.w < 0) {
      const double e = a.rhs[n + pc.z] - acc;
      if (lane == 0) a.res[n + pc.z] = e;
      local = fmax(local, fabs(e));
      nan |= e != e;
    } else if (lane == 0) {
      d.row_partial[pc.w] = acc;
    }
  }
  record_norm(a.norm, local, nan);
}

// the rows of A that were cut: their pieces' sums in order
__global__ void k_kkt_residual_combine(KktDev d, ResidualArgs a) {
  if (a.run && !*a.run) return;
  double local = 0.0;
  bool nan = false;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.row_combs; c += gridDim.x * blockDim.x) {
    const int4 cb = d.row_comb[c];
    double acc = 0.0;
    for (int k = 0; k < cb.z; ++k) acc += d.row_partial[cb.y + k];
    const double e = a.rhs[d.n + cb.x] - acc;
    a.res[d.n + cb.x] = e;
    local = fmax(local, fabs(e));
    nan |= e != e;
  }
  record_norm(a.norm, local, nan);
}

// rhs = [top (or 0); bottom], sol = rhs; the refinement record is cleared
__global__ void k_kkt_pack(int n, int m, const double* top, const double* bottom, double* rhs, double* sol,
                           KktRefine* rf) {
  if (blockIdx.x == 0 && threadIdx.x == 0) *rf = KktRefine{};
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n + m; t += gridDim.x * blockDim.x) {
    const double v = t < n ? (top ? top[t] : 0.0) : bottom[t - n];
    rhs[t] = v;
    sol[t] = v;
  }
}

// step r: runs when the previous step kept its candidate and the residual is not yet 0; cor = res
__global__ void k_kkt_begin(int count, int r, const double* res, double* cor, KktRefine* rf) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const bool prev = r == 0 || rf->acc[r - 1];
    rf->run[r] = prev && bits_to(rf->err[r]) > 0.0;
  }
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) cor[t] = res[t];
}

// the candidate sol + cor is kept when its residual is below half the current one
__global__ void k_kkt_accept(int count, int r, double* sol, const double* cor, double* res, const double* res2,
                             KktRefine* rf) {
  const bool keep = rf->run[r] && bits_to(rf->next[r]) < 0.5 * bits_to(rf->err[r]);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    rf->acc[r] = keep;
    rf->err[r + 1] = keep ? rf->next[r] : rf->err[r];
  }
  if (!keep) return;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
    sol[t] += cor[t];
    res[t] = res2[t];
  }
}

// dx = u, dy = -v (dx may be null)
__global__ void k_kkt_split(int n, int m, const double* w, double* dx, double* dy) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n + m; t += gridDim.x * blockDim.x) {
    if (t < n) {
      if (dx) dx[t] = w[t];
    } else {
      dy[t - n] = -w[t];
    }
  }
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

KktSystem::~KktSystem() {
  for (void* p : bufs_) cudaFree(p);
}

void KktSystem::build(const StdForm& f, const int* q_ptr_dev, const int* q_idx_dev, const double* q_val_dev,
                      const double* qdiag_dev, const int* col_ptr_dev, const int* row_idx_dev, const double* cval_dev,
                      const int* row_ptr_dev, const int* col_idx_dev, const double* rval_dev, const uint8_t* free_dev,
                      int* drop_count, int* fail, cudaStream_t st) {
  n_ = f.n;
  m_ = f.m;
  const int n = n_, m = m_, N = n + m;
  // pattern of K without its diagonal: Q's couplings among the columns, A between columns and rows
  std::vector<std::vector<int>> adj(N);
  for (int j = 0; j < n; ++j)
    for (int k = f.q_ptr[j]; k < f.q_ptr[j + 1]; ++k) {
      const int i = f.q_idx[k];
      if (i == j) continue;
      adj[j].push_back(i);
    }
  for (int j = 0; j < n; ++j)
    for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p) {
      adj[j].push_back(n + f.row_idx[p]);
      adj[n + f.row_idx[p]].push_back(j);
    }
  for (auto& l : adj) {
    std::sort(l.begin(), l.end());
    l.erase(std::unique(l.begin(), l.end()), l.end());
  }
  if (!sparse_analyze_graph(adj, 0, sym_))
    throw std::runtime_error("sparse L D L' of the order-" + std::to_string(N) + " KKT matrix needs more than " +
                             std::to_string(kMaxUpdates) + " rank-1 update terms");
  std::vector<int> q_slot(f.q_idx.size(), -1), a_slot(f.row_idx.size()), xs(n), ys(m);
  for (int j = 0; j < n; ++j)
    for (int k = f.q_ptr[j]; k < f.q_ptr[j + 1]; ++k)
      if (f.q_idx[k] > j) q_slot[k] = sparse_slot(sym_, f.q_idx[k], j);
  for (int j = 0; j < n; ++j)
    for (int p = f.col_ptr[j]; p < f.col_ptr[j + 1]; ++p) a_slot[p] = sparse_slot(sym_, n + f.row_idx[p], j);
  for (int j = 0; j < n; ++j) xs[j] = sparse_slot(sym_, j, j);
  for (int i = 0; i < m; ++i) ys[i] = sparse_slot(sym_, n + i, n + i);
  for (int v : q_slot)
    if (v < -1) throw std::runtime_error("KKT pattern: missing slot");
  for (int v : a_slot)
    if (v < 0) throw std::runtime_error("KKT pattern: missing slot");
  nq_ = static_cast<long long>(f.q_idx.size());
  na_ = static_cast<long long>(f.row_idx.size());
  std::vector<int8_t> sign(N, 1);
  for (int i = 0; i < m; ++i) sign[n + i] = -1;
  // a pivot only needs its sign: the drop threshold is 0
  factor_.upload(sym_, drop_count, fail, 0.0, st, &sign);
  fail_ = fail;
  drops_ = drop_count;
  d_.n = n;
  d_.m = m;
  d_.q_ptr = q_ptr_dev;
  d_.q_idx = q_idx_dev;
  d_.q_val = q_val_dev;
  d_.qdiag = qdiag_dev;
  d_.col_ptr = col_ptr_dev;
  d_.row_idx = row_idx_dev;
  d_.cval = cval_dev;
  d_.row_ptr = row_ptr_dev;
  d_.col_idx = col_idx_dev;
  d_.rval = rval_dev;
  d_.free_col = free_dev;
  d_.q_slot = put(bufs_, q_slot, st);
  d_.a_slot = put(bufs_, a_slot, st);
  d_.xdiag_slot = put(bufs_, xs, st);
  d_.ydiag_slot = put(bufs_, ys, st);
  d_.V = factor_.values();
  d_.diag = factor_.assembled_diag();
  {
    int slots = 0;
    const SparsePieces rp = row_pieces(f.row_ptr, &slots);
    static_assert(sizeof(SparsePiece) == sizeof(int4) && sizeof(SparseCombine) == sizeof(int4), "piece layout");
    d_.row_piece = reinterpret_cast<const int4*>(put(bufs_, rp.piece, st));
    d_.row_pieces = static_cast<int>(rp.piece.size());
    d_.row_comb = reinterpret_cast<const int4*>(put(bufs_, rp.comb, st));
    d_.row_combs = static_cast<int>(rp.comb.size());
    d_.row_partial = put(bufs_, std::vector<double>(std::max(1, slots), 0.0), st);
  }
  const std::vector<double> zeros(static_cast<size_t>(N), 0.0);
  rhs_ = put(bufs_, zeros, st);
  sol_ = put(bufs_, zeros, st);
  res_ = put(bufs_, zeros, st);
  cor_ = put(bufs_, zeros, st);
  res2_ = put(bufs_, zeros, st);
  const std::vector<unsigned char> rf(sizeof(KktRefine), 0);
  refine_ = put(bufs_, rf, st);
  SOV_CUDA(cudaStreamSynchronize(st));  // host vectors above go out of scope
}

bool KktSystem::assemble_and_factor(bool start, const double* x, const double* s, cudaStream_t st, int* launches) {
  start_ = start;
  x_ = x;
  s_ = s;
  const int N = n_ + m_;
  const int grid = blocks_for(std::max<long long>(std::max(nq_, na_), N));
  // delta never falls back below a value that was needed once (qp_interior_point.cpp:459-463)
  for (double delta = std::max(delta_, kDeltaMin); delta <= kDeltaMax; delta *= 100.0) {
    SOV_CUDA(cudaMemsetAsync(d_.V, 0, sizeof(double) * (N + sym_.nnz_l), st));
    SOV_CUDA(cudaMemsetAsync(fail_, 0, sizeof(int), st));
    SOV_CUDA(cudaMemsetAsync(drops_, 0, sizeof(int), st));
    k_kkt_assemble<<<grid, kKktThreads, 0, st>>>(d_, x, s, start ? 1 : 0, delta);
    SOV_LAUNCH_CHECK();
    factor_.factor(st, launches);
    SOV_CUDA(cudaMemcpyAsync(&flags_h_[0], fail_, sizeof(int), cudaMemcpyDeviceToHost, st));
    SOV_CUDA(cudaMemcpyAsync(&flags_h_[1], drops_, sizeof(int), cudaMemcpyDeviceToHost, st));
    SOV_CUDA(cudaStreamSynchronize(st));
    if (launches) *launches += 1;
    ++factorizations_;
    if (!flags_h_[0] && !flags_h_[1]) {
      delta_ = delta;
      return true;
    }
  }
  // no delta up to 1e-5 gives every pivot its sign: the factorization failed
  static const int one = 1;
  SOV_CUDA(cudaMemcpyAsync(fail_, &one, sizeof(int), cudaMemcpyHostToDevice, st));
  SOV_CUDA(cudaStreamSynchronize(st));
  return false;
}

void KktSystem::residual(const double* w, const double* c, double* res, unsigned long long* norm, const int* run,
                         cudaStream_t st) {
  const ResidualArgs a{x_, s_, start_ ? 1 : 0, rhs_, w, c, res, norm, run};
  const long long work = std::max<long long>(n_, 32LL * d_.row_pieces);
  k_kkt_residual<<<blocks_for(work), kKktThreads, 0, st>>>(d_, a);
  if (d_.row_combs) k_kkt_residual_combine<<<blocks_for(d_.row_combs), kKktThreads, 0, st>>>(d_, a);
}

void KktSystem::solve_refined(const double* top, const double* bottom, double* dx, double* dy, cudaStream_t st,
                              int* launches) {
  const int n = n_, m = m_, N = n + m;
  const int g = blocks_for(N);
  KktRefine* rf = static_cast<KktRefine*>(refine_);
  k_kkt_pack<<<g, kKktThreads, 0, st>>>(n, m, top, bottom, rhs_, sol_, rf);
  factor_.solve(sol_, st, launches);
  residual(sol_, nullptr, res_, &rf->err[0], nullptr, st);
  for (int r = 0; r < kKktRefineSteps; ++r) {
    k_kkt_begin<<<g, kKktThreads, 0, st>>>(N, r, res_, cor_, rf);
    factor_.solve(cor_, st, launches, &rf->run[r]);
    residual(sol_, cor_, res2_, &rf->next[r], &rf->run[r], st);
    k_kkt_accept<<<g, kKktThreads, 0, st>>>(N, r, sol_, cor_, res_, res2_, rf);
  }
  k_kkt_split<<<g, kKktThreads, 0, st>>>(n, m, sol_, dx, dy);
  SOV_LAUNCH_CHECK();
  if (launches) *launches += (3 + 3 * kKktRefineSteps) + (d_.row_combs ? 1 + kKktRefineSteps : 0);
}

void KktSystem::solve_newton(double* r1_dx, const double* rp, double* dy, cudaStream_t st, int* launches) {
  solve_refined(r1_dx, rp, r1_dx, dy, st, launches);
}

void KktSystem::solve_normal(double* z, cudaStream_t st, int* launches) {
  solve_refined(nullptr, z, nullptr, z, st, launches);
}

}  // namespace sov
