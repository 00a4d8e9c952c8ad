// engine.cu -- single-problem GPU interior-point engine.
//
// The iteration of solve_ipm (solver/lp/src/interior_point.cpp:454-740) and of the generic QP path
// solve_qp_ipm (solver/qp/src/qp_interior_point.cpp:2848-3116, diagonal Hessians), with all
// vectors resident in HBM. Per iteration the host reads one IpmScalars struct (residual norms,
// mu, gap, the previous step lengths) and takes the reference's decisions: best-iterate
// bookkeeping, the history samples and the stopping test. Everything else is stream-ordered
// device work: assembly of A D A', factorization, two Newton solves, ratio tests, update.
//
// Normal-equation backends:
//   dense FP64    blocked Cholesky + dataflow triangular solves (the plain FP64 engine)
//   dense mixed   FP32 Cholesky as the preconditioner of FP64 PCG on the exact normal operator;
//                 an iteration whose PCG does not converge is refactored in FP64
//   band          banded LDL^T, natural order, for small half-bandwidths
//   sparse        sparse LDL^T after a minimum-degree order, level-scheduled on the GPU
// A QP whose Hessian couples variables takes its Newton step from y-space normal equations with a
// dense H = Q + X^-1 S (up to kCoupledMaxColumns columns), or from the quasi-definite KKT system
// [H + delta I, A'; A, -delta I] as a sparse LDL^T (kkt.cuh) -- the reference's QpKkt form.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "band.cuh"
#include "common.cuh"
#include "dense.cuh"
#include "engine.hpp"
#include "xband.hpp"
#include "ipm_kernels.cuh"
#include "kkt.cuh"
#include "sparse.hpp"
#include "sparse_gpu.cuh"

namespace sov {
namespace {

// Device buffers of one solve are stream-ordered allocations on the solve's stream (the default
// memory pool of the device, kept cached up to kPoolKeep bytes): concurrent solves on other
// streams neither pay cudaMalloc nor wait on the device-wide synchronisation of cudaFree.
thread_local cudaStream_t tl_alloc_stream = nullptr;  // set by Engine::setup for its buffers
constexpr uint64_t kPoolKeep = uint64_t(4) << 30;

void keep_pool_memory() {
  static std::mutex mu;
  static std::vector<int> done;
  int dev = 0;
  SOV_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  if (std::find(done.begin(), done.end(), dev) != done.end()) return;
  cudaMemPool_t pool;
  SOV_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
  uint64_t keep = kPoolKeep;
  SOV_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  done.push_back(dev);
}

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t st = nullptr;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  void alloc(size_t count) {
    release();
    n = count;
    st = tl_alloc_stream;
    if (count) SOV_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), sizeof(T) * count, st));
  }
  void zero(cudaStream_t st) {
    if (n) SOV_CUDA(cudaMemsetAsync(p, 0, sizeof(T) * n, st));
  }
  void upload(const T* h, size_t count, cudaStream_t st) {
    if (count) SOV_CUDA(cudaMemcpyAsync(p, h, sizeof(T) * count, cudaMemcpyHostToDevice, st));
  }
  void release() {
    if (p) cudaFreeAsync(p, st);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// Pinned 256-byte slots for the few scalars a solve reads back every iteration, from one pinned
// block shared by all solves of the process (pinning and unpinning per solve would serialise
// concurrent solves).
class PinnedSlots {
 public:
  void* acquire() {
    std::lock_guard<std::mutex> g(mu_);
    if (free_.empty()) {
      unsigned char* block = nullptr;
      SOV_CUDA(cudaMallocHost(&block, kSlot * kPerBlock));
      for (int k = kPerBlock - 1; k >= 0; --k) free_.push_back(block + kSlot * k);
    }
    void* p = free_.back();
    free_.pop_back();
    return p;
  }
  void release(void* p) {
    std::lock_guard<std::mutex> g(mu_);
    free_.push_back(p);
  }

 private:
  static constexpr size_t kSlot = 256;
  static constexpr int kPerBlock = 256;
  std::mutex mu_;
  std::vector<void*> free_;
};
PinnedSlots g_pinned_slots;

struct PinnedScalars {
  IpmScalars* h = nullptr;
  PinnedScalars() {
    static_assert(sizeof(IpmScalars) <= 256, "scalar block larger than a pinned slot");
    h = static_cast<IpmScalars*>(g_pinned_slots.acquire());
  }
  ~PinnedScalars() { g_pinned_slots.release(h); }
};

// -------------------------------------------------------------------------------------------
// PCG helpers (single CTA; the dense path has m <= 8192)
// -------------------------------------------------------------------------------------------
struct PcgScalars {
  double rz, rr, bb, alpha, beta;
};

__global__ void __launch_bounds__(1024) k_pcg_init(int m, const double* rhs, double* x, double* r, double* w,
                                                   PcgScalars* ps) {
  __shared__ double scratch[4 * 32];
  double bb = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const double v = rhs[i];
    x[i] = 0.0;
    r[i] = v;
    w[i] = v;
    bb += v * v;
  }
  double v4[4] = {bb, 0, 0, 0};
  const int ops[4] = {0, 0, 0, 0};
  block_reduce<4>(v4, ops, scratch);
  if (threadIdx.x == 0) {
    ps->bb = v4[0];
    ps->rr = v4[0];
  }
}

// after w = P^-1 r: rz_new = r.w; beta = rz_new / rz (first: beta = 0); p = w + beta p
__global__ void __launch_bounds__(1024) k_pcg_direction(int m, const double* r, const double* w, double* p,
                                                        PcgScalars* ps, int first) {
  __shared__ double scratch[4 * 32];
  __shared__ double beta_s;
  double rz = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) rz += r[i] * w[i];
  double v4[4] = {rz, 0, 0, 0};
  const int ops[4] = {0, 0, 0, 0};
  block_reduce<4>(v4, ops, scratch);
  if (threadIdx.x == 0) {
    const double beta = first ? 0.0 : v4[0] / ps->rz;
    ps->beta = beta;
    ps->rz = v4[0];
    beta_s = beta;
  }
  __syncthreads();
  const double beta = beta_s;
  for (int i = threadIdx.x; i < m; i += blockDim.x) p[i] = w[i] + beta * (first ? 0.0 : p[i]);
}

// q = M p given; alpha = rz / p.q; x += alpha p; r -= alpha q; w = r (to be preconditioned)
__global__ void __launch_bounds__(1024) k_pcg_step(int m, const double* p, const double* q, double* x, double* r,
                                                   double* w, PcgScalars* ps) {
  __shared__ double scratch[4 * 32];
  __shared__ double alpha_s;
  double pq = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) pq += p[i] * q[i];
  double v4[4] = {pq, 0, 0, 0};
  const int ops[4] = {0, 0, 0, 0};
  block_reduce<4>(v4, ops, scratch);
  if (threadIdx.x == 0) {
    const double a = v4[0] != 0.0 ? ps->rz / v4[0] : 0.0;
    ps->alpha = a;
    alpha_s = a;
  }
  __syncthreads();
  const double a = alpha_s;
  double rr = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    x[i] += a * p[i];
    const double ri = r[i] - a * q[i];
    r[i] = ri;
    w[i] = ri;
    rr += ri * ri;
  }
  double u4[4] = {rr, 0, 0, 0};
  block_reduce<4>(u4, ops, scratch);
  if (threadIdx.x == 0) ps->rr = u4[0];
}

// -------------------------------------------------------------------------------------------

class Engine {
 public:
  Engine(const sov_model& model, const StdForm& f, const sov_options& opt, cudaStream_t st, EngineStats* stats,
         bool mehrotra_start = false)
      : model_(model), f_(f), opt_(opt), st_(st), stats_(stats), mehrotra_start_(mehrotra_start) {}

  void run(sov_result* r);

 private:
  void setup();
  void assemble_and_factor(int mode);
  bool newton_solve();  // z -> dy in place
  void read_scalars();
  void publish(const DevBuf<double>& x, const DevBuf<double>& y, const DevBuf<double>& s, int status, int iteration,
               double gap, double pres, double dres, const std::string& msg, sov_result* r);
  std::string describe() const;

  const sov_model& model_;
  const StdForm& f_;
  sov_options opt_;
  cudaStream_t st_;
  EngineStats* stats_;
  int launches_ = 0;

  // device data
  DevBuf<int> row_ptr_, col_idx_, col_ptr_, row_idx_;
  DevBuf<double> rval_, cval_, b_, c_, qdiag_;
  DevBuf<uint8_t> free_;
  DevBuf<double> x_, y_, s_, dx_, ds_, dxa_, dsa_, rp_, rd_, z_, bx_, by_, bs_;
  DevBuf<double> cx_, cy_, cs_;  // iterate captured at the start of iteration opt_.ipm_iterate_at
  bool captured_ = false;
  DevBuf<double> partials_;
  DevBuf<unsigned> counter_;
  DevBuf<IpmScalars> sc_;
  PinnedScalars hs_;
  IpmDev dev_{};

  // factorization
  enum Backend { kDense64, kDenseMixed, kBand, kSparse, kKkt } backend_ = kDense64;
  // sparse quasi-definite KKT system of a coupled-Hessian QP (kKkt)
  std::unique_ptr<KktSystem> kkt_;
  // sparse L D L' (kSparse): symbolic analysis on the host, numeric factor and solves on the GPU
  SparseSymbolic sym_;
  SparseFactor sparse_;
  DevBuf<int64_t> sp_target_;
  DevBuf<int> sp_ptr_, sp_col_;
  DevBuf<double> sp_w_;
  AssemblyDev spd_{};
  int mp_ = 0, nb_ = 0, kd_ = 0;
  AssemblyMap am_;
  DevBuf<int64_t> am_target_;
  DevBuf<int> am_ptr_, am_col_, am_diag_;
  DevBuf<double> am_w_;
  AssemblyDev amd_{};
  DevBuf<double> M64_, Linv64_;
  DevBuf<float> M32_, Linv32_;
  DevBuf<double> diag_, band_, dinv_;
  DevBuf<unsigned> flags_;
  DevBuf<int> err_;
  unsigned epoch_ = 0;
  DenseSystem<double> ds64_{};
  DenseSystem<float> ds32_{};
  BandSystem bandsys_{};
  int last_mode_ = kWeightLp;
  bool fp64_ready_ = false;  // FP64 factor of the current iteration exists (mixed fallback)
  // PCG work
  DevBuf<double> pcg_x_, pcg_r_, pcg_w_, pcg_p_, pcg_q_, pcg_tmp_;
  DevBuf<PcgScalars> pcg_s_;
  PcgScalars* pcg_h_ = nullptr;
  int pcg_iterations_ = 0, fp64_fallbacks_ = 0, factorizations_ = 0;
  // mixed precision stops paying once the FP32 factor needs many PCG steps per solve (the normal
  // matrix only gets worse conditioned as the iterates approach the boundary): from the next
  // factorization on, the engine factors in FP64
  static constexpr int kPcgSwitch = 12;
  static constexpr int kWarmGiveUp = 40;  // iterations a supplied start gets before the default restart
  static constexpr int kCoupledMaxColumns = 16384;  // dense H of a coupled-Hessian QP: at most 2 GB
  // automatic choice of the sparse KKT system for a coupled-Hessian QP: a KKT order of at least
  // this and at most kKktSparseCoupling off-diagonal Q entries per column
  static constexpr int kKktAutoOrder = 2048;
  static constexpr int kKktSparseCoupling = 32;
  static constexpr int kDenseMaxOrder = 16384;      // dense normal matrix: at most 2 GB
  bool to_fp64_ = false;
  bool sparse_refused_ = false;  // the sparse factor was asked for but is nearly dense: dense instead
  // x-space QP
  XSpace xs_;
  bool xspace_ = false;
  int order_ = 0;  // order of the factored system: m (y-space) or structural columns (x-space)
  DevBuf<int> slack_of_row_;
  DevBuf<double> coltmp_;
  DevBuf<int> row_piece_, row_comb_;
  DevBuf<double> row_partial_;
  static constexpr int kLongRow = 512;
  DevBuf<double> sigma_, tr_, dyv_;
  // QP with a coupled Hessian: dense H = Q + diag(h) (order n, padded to nph_), its factor, and
  // Y = H^-1 A' for the reduced system M = A H^-1 A'
  bool coupled_ = false;
  int nph_ = 0, nbh_ = 0;
  DevBuf<int> q_ptr_, q_idx_;
  DevBuf<double> q_val_, qdense_, hmat_, hlinv_, hdiag_, ymat_, hvec_;
  DevBuf<unsigned> hflags_;
  DenseSystem<double> dsh_{};
  void coupled_newton(int mode);
  // QP second attempt: Mehrotra's starting point in place of the default one
  bool mehrotra_start_ = false;
  void mehrotra_qp_start();
};

void Engine::setup() {
  tl_alloc_stream = st_;
  keep_pool_memory();
  const int m = f_.m, n = f_.n;
  row_ptr_.alloc(m + 1);
  row_ptr_.upload(f_.row_ptr.data(), m + 1, st_);
  col_idx_.alloc(f_.nnz());
  col_idx_.upload(f_.col_idx.data(), f_.nnz(), st_);
  rval_.alloc(f_.nnz());
  rval_.upload(f_.rval.data(), f_.nnz(), st_);
  col_ptr_.alloc(n + 1);
  col_ptr_.upload(f_.col_ptr.data(), n + 1, st_);
  row_idx_.alloc(f_.nnz());
  row_idx_.upload(f_.row_idx.data(), f_.nnz(), st_);
  cval_.alloc(f_.nnz());
  cval_.upload(f_.val.data(), f_.nnz(), st_);
  b_.alloc(m);
  b_.upload(f_.b.data(), m, st_);
  c_.alloc(n);
  c_.upload(f_.c.data(), n, st_);
  if (f_.qp) {
    qdiag_.alloc(n);
    qdiag_.upload(f_.qdiag.data(), n, st_);
    free_.alloc(n);
    free_.upload(f_.free_col.data(), n, st_);
  }
  for (DevBuf<double>* v : {&x_, &s_, &dx_, &ds_, &dxa_, &dsa_, &rd_, &bx_, &bs_}) v->alloc(n);
  for (DevBuf<double>* v : {&y_, &rp_, &by_}) v->alloc(m);
  partials_.alloc(8 * 1184);
  counter_.alloc(1);
  counter_.zero(st_);
  sc_.alloc(1);
  sc_.zero(st_);
  err_.alloc(1);
  err_.zero(st_);

  // x-space for QPs whose rows all carry slacks and whose structural columns have Q_jj > 0
  xs_ = analyze_xspace(f_);
  if (opt_.factorization == SOV_FACTOR_XSPACE && !(f_.qp && xs_.eligible))
    throw std::runtime_error("x-space factorization needs a QP whose rows are all inequalities and whose structural "
                             "columns all have Q_jj > 0");
  xspace_ = opt_.factorization == SOV_FACTOR_XSPACE;
  coupled_ = f_.qp && !f_.q_diagonal;
  // a free column without curvature (Q_jj no more than the 1e-14 every column carries) makes H^-1
  // blow up in the normal equations; the KKT system takes it with the pivot Q_jj + delta
  bool flat_free = false;
  if (f_.qp)
    for (int j = 0; j < n && !flat_free; ++j) flat_free = f_.free_col[j] && !(f_.qdiag[j] > 1e-12);
  bool want_kkt = flat_free;
  if (flat_free && opt_.factorization != SOV_FACTOR_AUTO && opt_.factorization != SOV_FACTOR_SPARSE)
    throw std::runtime_error("a free variable without curvature (Q_jj = 0) needs the KKT system: factorization "
                             "AUTO or SPARSE");
  if (coupled_) {
    // the y-space system needs H^-1 of the coupled Hessian (dense H, FP64); the KKT system does not
    if (opt_.factorization == SOV_FACTOR_BANDED)
      throw std::runtime_error("banded factorization needs a separable Hessian; this QP couples variables in Q");
    const long long q_off = static_cast<long long>(f_.q_idx.size()) - n;
    want_kkt = want_kkt || opt_.factorization == SOV_FACTOR_SPARSE || n > kCoupledMaxColumns ||
               (opt_.factorization == SOV_FACTOR_AUTO && n + m >= kKktAutoOrder &&
                q_off <= static_cast<long long>(kKktSparseCoupling) * n);
  }
  order_ = xspace_ ? f_.n_struct : m;
  // backend choice: band when the half-bandwidth is small, else dense (mixed or FP64)
  kd_ = xspace_ ? xs_.kd : normal_bandwidth(f_);
  const bool auto_pick = opt_.factorization == SOV_FACTOR_AUTO || opt_.factorization == SOV_FACTOR_XSPACE;
  const bool want_band =
      !coupled_ && (opt_.factorization == SOV_FACTOR_BANDED || (auto_pick && kd_ <= kBandMax && order_ > 256));
  // sparse L D L' when asked for, or when the normal matrix is beyond the dense factorization
  const bool want_sparse = !want_band && !xspace_ && !coupled_ &&
                           (opt_.factorization == SOV_FACTOR_SPARSE ||
                            (opt_.factorization == SOV_FACTOR_AUTO && order_ > kDenseMaxOrder));
  if (opt_.factorization == SOV_FACTOR_SPARSE && xspace_)
    throw std::runtime_error("the sparse factorization takes the y-space normal equations or the KKT system, not "
                             "the x-space system");
  // a normal matrix whose sparse factor would need more rank-1 terms than the update schedule
  // holds is nearly dense: it is factored densely when it fits
  bool sparse_ok = want_sparse && sparse_analyze(f_, 0, sym_);
  if (want_sparse && !sparse_ok) {
    if (order_ > kDenseMaxOrder)
      throw std::runtime_error("sparse L D L' of the order-" + std::to_string(order_) +
                               " normal matrix needs more than " + std::to_string(kMaxUpdates) +
                               " rank-1 update terms");
    sparse_refused_ = true;
  }
  if (want_kkt) {
    backend_ = kKkt;
  } else if (sparse_ok) {
    backend_ = kSparse;
  } else if (want_band) {
    if (kd_ > kBandMax) throw std::runtime_error("banded factorization requested but half-bandwidth " +
                                                 std::to_string(kd_) + " exceeds " + std::to_string(kBandMax));
    backend_ = kBand;
  } else {
    if (order_ > kDenseMaxOrder) throw std::runtime_error("normal matrix of order " + std::to_string(order_) +
                                                 " is too large for the dense factorization (band width " +
                                                 std::to_string(kd_) + ")");
    // the x-space system has no matrix-free PCG operator: it is factored in FP64
    backend_ = (opt_.precision == SOV_PRECISION_MIXED && !xspace_ && !coupled_) ? kDenseMixed : kDense64;
  }
  if (backend_ == kKkt) {
    z_.alloc(std::max(1, m));
    z_.zero(st_);
  } else if (backend_ == kSparse) {
    std::vector<int64_t> tg(sym_.asm_target.begin(), sym_.asm_target.end());
    sp_target_.alloc(tg.size());
    sp_target_.upload(tg.data(), tg.size(), st_);
    sp_ptr_.alloc(sym_.asm_ptr.size());
    sp_ptr_.upload(sym_.asm_ptr.data(), sym_.asm_ptr.size(), st_);
    sp_col_.alloc(sym_.asm_col.size());
    sp_col_.upload(sym_.asm_col.data(), sym_.asm_col.size(), st_);
    sp_w_.alloc(sym_.asm_w.size());
    sp_w_.upload(sym_.asm_w.data(), sym_.asm_w.size(), st_);
    spd_ = AssemblyDev{sp_target_.p, sp_ptr_.p, sp_col_.p, sp_w_.p, nullptr, static_cast<int>(tg.size())};
    z_.alloc(order_);
    z_.zero(st_);
  } else if (backend_ == kBand) {
    am_ = xspace_ ? build_assembly_xspace_band(f_, xs_) : build_assembly_band(f_, kd_);
    band_.alloc(static_cast<size_t>(kBandMax + 1) * order_);
    band_.zero(st_);
    dinv_.alloc(order_);
    diag_.alloc(order_);
    z_.alloc(order_);
    z_.zero(st_);
    bandsys_ = BandSystem{band_.p, dinv_.p, diag_.p, order_, kd_, nullptr, nullptr};
  } else {
    nb_ = ceil_div(order_, kNB);
    mp_ = nb_ * kNB;
    am_ = xspace_ ? build_assembly_xspace(f_, xs_, mp_) : build_assembly_dense(f_, mp_);
    diag_.alloc(order_);
    flags_.alloc(nb_ + 1);  // + the factor's ticket counter
    flags_.zero(st_);
    z_.alloc(mp_);
    z_.zero(st_);
    if (backend_ == kDenseMixed) {
      M32_.alloc(static_cast<size_t>(mp_) * mp_);
      Linv32_.alloc(static_cast<size_t>(nb_) * kNB * kNB);
      for (DevBuf<double>* v : {&pcg_x_, &pcg_r_, &pcg_w_, &pcg_p_, &pcg_q_}) {
        v->alloc(mp_);
        v->zero(st_);
      }
      pcg_tmp_.alloc(n);
      pcg_s_.alloc(1);
      pcg_h_ = static_cast<PcgScalars*>(g_pinned_slots.acquire());
    }
  }
  if (coupled_ || backend_ == kKkt) {
    q_ptr_.alloc(n + 1);
    q_ptr_.upload(f_.q_ptr.data(), n + 1, st_);
    q_idx_.alloc(f_.q_idx.size());
    q_idx_.upload(f_.q_idx.data(), f_.q_idx.size(), st_);
    q_val_.alloc(f_.q_val.size());
    q_val_.upload(f_.q_val.data(), f_.q_val.size(), st_);
  }
  if (backend_ == kKkt) {
    hvec_.alloc(n);
    hvec_.zero(st_);
  } else if (coupled_) {
    nbh_ = ceil_div(n, kNB);
    nph_ = nbh_ * kNB;
    // dense Q (column-major, both triangles) with the padding's diagonal 1
    std::vector<double> qd(static_cast<size_t>(nph_) * nph_, 0.0);
    for (int j = 0; j < n; ++j)
      for (int k = f_.q_ptr[j]; k < f_.q_ptr[j + 1]; ++k) qd[static_cast<size_t>(j) * nph_ + f_.q_idx[k]] = f_.q_val[k];
    for (int j = n; j < nph_; ++j) qd[static_cast<size_t>(j) * nph_ + j] = 1.0;
    qdense_.alloc(qd.size());
    qdense_.upload(qd.data(), qd.size(), st_);
    hmat_.alloc(qd.size());
    hlinv_.alloc(static_cast<size_t>(nbh_) * kNB * kNB);
    hdiag_.alloc(n);
    hflags_.alloc(nbh_ + 1);
    hflags_.zero(st_);
    ymat_.alloc(static_cast<size_t>(nph_) * std::max(1, m));
    hvec_.alloc(nph_);
    hvec_.zero(st_);
  }
  if (xspace_) {
    slack_of_row_.alloc(m);
    slack_of_row_.upload(xs_.slack_of_row.data(), m, st_);
    sigma_.alloc(m);
    sigma_.upload(xs_.sigma.data(), m, st_);
    tr_.alloc(m);
    dyv_.alloc(m);
  }
  if (backend_ == kSparse) {
    IpmScalars* sc0 = sc_.p;
    sparse_.upload(sym_, &sc0->drops, &sc0->fail, 1e-13, st_);
  }
  am_target_.alloc(am_.target.size());
  am_target_.upload(am_.target.data(), am_.target.size(), st_);
  am_ptr_.alloc(am_.ptr.size());
  am_ptr_.upload(am_.ptr.data(), am_.ptr.size(), st_);
  am_col_.alloc(am_.col.size());
  am_col_.upload(am_.col.data(), am_.col.size(), st_);
  am_w_.alloc(am_.w.size());
  am_w_.upload(am_.w.data(), am_.w.size(), st_);
  am_diag_.alloc(am_.diag_target.size());
  am_diag_.upload(am_.diag_target.data(), am_.diag_target.size(), st_);
  amd_ = AssemblyDev{am_target_.p, am_ptr_.p, am_col_.p, am_w_.p, am_diag_.p, static_cast<int>(am_.target.size())};

  IpmScalars* sc = sc_.p;
  int* fail_ptr = &sc->fail;
  int* drop_ptr = &sc->drops;
  if (backend_ == kBand) {
    bandsys_.drop_count = drop_ptr;
    bandsys_.fail = fail_ptr;
  } else {
    ds32_ = DenseSystem<float>{M32_.p, Linv32_.p, diag_.p, order_, mp_, nb_, drop_ptr, fail_ptr, flags_.p, flags_.p + nb_, 1e-6};
  }
  if (backend_ == kKkt) {
    kkt_ = std::make_unique<KktSystem>();
    kkt_->build(f_, q_ptr_.p, q_idx_.p, q_val_.p, qdiag_.p, col_ptr_.p, row_idx_.p, cval_.p, row_ptr_.p, col_idx_.p,
                rval_.p, free_.p, drop_ptr, fail_ptr, st_);
  } else if (coupled_) {
    dsh_ = DenseSystem<double>{hmat_.p, hlinv_.p, hdiag_.p, n, nph_, nbh_, drop_ptr, fail_ptr, hflags_.p,
                               hflags_.p + nbh_, 1e-13};
  }

  dev_.m = m;
  dev_.n = n;
  dev_.row_ptr = row_ptr_.p;
  dev_.col_idx = col_idx_.p;
  dev_.rval = rval_.p;
  dev_.col_ptr = col_ptr_.p;
  dev_.row_idx = row_idx_.p;
  dev_.cval = cval_.p;
  dev_.b = b_.p;
  dev_.c = c_.p;
  dev_.qdiag = qdiag_.p;
  dev_.free_col = free_.p;
  dev_.q_ptr = q_ptr_.p;
  dev_.q_idx = q_idx_.p;
  dev_.q_val = q_val_.p;
  dev_.q_coupled = coupled_ ? 1 : 0;
  dev_.qp = f_.qp ? 1 : 0;
  dev_.has_quadratic = f_.has_quadratic ? 1 : 0;
  int n_bounded = 0;
  for (int j = 0; j < n; ++j) n_bounded += f_.free_col[j] ? 0 : 1;
  dev_.comp_count = f_.qp ? std::max(1, n_bounded) : n;
  double bmax = 0.0, cmax = 0.0;
  for (double v : f_.b) bmax = std::max(bmax, std::abs(v));
  for (double v : f_.c) cmax = std::max(cmax, std::abs(v));
  dev_.bnorm = std::max(1.0, bmax);
  dev_.cnorm = std::max(1.0, cmax);
  dev_.objective_offset = f_.objective_offset;
  dev_.tau = opt_.fraction_to_boundary;
  dev_.x = x_.p;
  dev_.y = y_.p;
  dev_.s = s_.p;
  dev_.dx = dx_.p;
  dev_.ds = ds_.p;
  dev_.dxa = dxa_.p;
  dev_.dsa = dsa_.p;
  dev_.rp = rp_.p;
  dev_.rd = rd_.p;
  dev_.z = z_.p;
  dev_.dy = xspace_ ? dyv_.p : z_.p;
  dev_.xspace = xspace_ ? 1 : 0;
  dev_.nx = f_.n_struct;
  dev_.slack_of_row = slack_of_row_.p;
  dev_.sigma = sigma_.p;
  dev_.tr = tr_.p;
  dev_.sc = sc_.p;
  // rows of at least kLongRow entries on average: a CTA per row, column terms computed once; a
  // row longer than a piece: the row kernels walk pieces
  if (!xspace_ && m > 0 && static_cast<long long>(f_.nnz()) >= static_cast<long long>(kLongRow) * m) {
    dev_.row_block = 1;
    coltmp_.alloc(n);
    dev_.coltmp = coltmp_.p;
  }
  int longest = 0;
  for (int i = 0; i < m; ++i) longest = std::max(longest, f_.row_ptr[i + 1] - f_.row_ptr[i]);
  if (!xspace_ && longest > kSparsePiece && dev_.row_block == 0) {
    int slots = 0;
    const SparsePieces rp = row_pieces(f_.row_ptr, &slots);
    static_assert(sizeof(SparsePiece) == sizeof(int4) && sizeof(SparseCombine) == sizeof(int4), "piece layout");
    row_piece_.alloc(4 * rp.piece.size());
    row_piece_.upload(reinterpret_cast<const int*>(rp.piece.data()), 4 * rp.piece.size(), st_);
    row_comb_.alloc(4 * rp.comb.size());
    row_comb_.upload(reinterpret_cast<const int*>(rp.comb.data()), 4 * rp.comb.size(), st_);
    row_partial_.alloc(std::max(1, slots));
    dev_.row_piece = reinterpret_cast<const int4*>(row_piece_.p);
    dev_.row_pieces = static_cast<int>(rp.piece.size());
    dev_.row_comb = reinterpret_cast<const int4*>(row_comb_.p);
    dev_.row_combs = static_cast<int>(rp.comb.size());
    dev_.row_partial = row_partial_.p;
    SOV_CUDA(cudaStreamSynchronize(st_));  // rp goes out of scope
  }
  dev_.partials = partials_.p;
  dev_.counter = counter_.p;
}

void Engine::assemble_and_factor(int mode) {
  last_mode_ = mode;
  const double reg = 1e-12;  // kNormalEqRegularization (interior_point.cpp:103)
  ++factorizations_;
  fp64_ready_ = false;
  if (to_fp64_ && backend_ == kDenseMixed) backend_ = kDense64;
  // x-space: K = A_x' Theta A_x (+ diag Q + H after assembly); start system: Theta = 1, diag 1
  const int amode = xspace_ ? (mode == kWeightOnes ? kWeightOnes : kWeightTheta) : mode;
  if (backend_ == kKkt) {
    // a failure leaves the fail flag set: the iteration loop stops with the factorization error
    kkt_->assemble_and_factor(mode == kWeightOnes, x_.p, s_.p, st_, &launches_);
    if (stats_) stats_->factor_flops += kkt_->flops();
    return;
  }
  if (backend_ == kSparse) {
    SOV_CUDA(cudaMemsetAsync(sparse_.values(), 0, sizeof(double) * (order_ + sparse_.nnz_l()), st_));
    launch_assemble<double>(spd_, x_.p, s_.p, qdiag_.p, free_.p, mode, reg, sparse_.values(), sparse_.assembled_diag(),
                            order_, 0, st_);
    sparse_.factor(st_, &launches_);
    launches_ += 2;
    if (stats_) stats_->factor_flops += sym_.flops;
    return;
  }
  if (backend_ == kBand) {
    launch_assemble<double>(amd_, x_.p, s_.p, qdiag_.p, free_.p, amode, reg, band_.p, diag_.p, order_, -order_, st_);
    if (xspace_) launch_xspace_diag(dev_, mode == kWeightOnes ? 0 : 1, band_.p, -1, diag_.p, st_);
    band_factor(bandsys_, st_, &launches_);
    launches_ += xspace_ ? 2 : 1;
    if (stats_) {
      const double kd = kd_;
      stats_->factor_flops += order_ * (kd * kd + 2.0 * kd);
    }
    return;
  }
  if (backend_ == kDense64) {
    if (!M64_.p) {
      M64_.alloc(static_cast<size_t>(mp_) * mp_);
      Linv64_.alloc(static_cast<size_t>(nb_) * kNB * kNB);
      ds64_ = DenseSystem<double>{M64_.p, Linv64_.p, diag_.p, order_, mp_, nb_, &sc_.p->drops, &sc_.p->fail, flags_.p, flags_.p + nb_, 1e-13};
    }
    if (coupled_ && mode != kWeightOnes) {
      // H = Q + diag(h), factored; Y = H^-1 A'; M = A Y + reg I, factored (the starting-point
      // system has H = I and takes the ordinary assembly below)
      SOV_CUDA(cudaMemcpyAsync(hmat_.p, qdense_.p, sizeof(double) * static_cast<size_t>(nph_) * nph_,
                               cudaMemcpyDeviceToDevice, st_));
      launch_hessian_diag(dev_, false, hmat_.p, nph_, hdiag_.p, st_);
      dense_cholesky<double>(dsh_, st_, &launches_);
      SOV_CUDA(cudaMemsetAsync(ymat_.p, 0, sizeof(double) * static_cast<size_t>(nph_) * std::max(1, f_.m), st_));
      launch_rows_to_columns(dev_, ymat_.p, nph_, st_);
      for (int i = 0; i < f_.m; ++i)
        dense_solve<double>(dsh_, ymat_.p + static_cast<size_t>(i) * nph_, epoch_, err_.p, st_, &launches_);
      launch_dense_clear<double>(M64_.p, order_, mp_, st_);
      launch_form_normal(dev_, ymat_.p, nph_, M64_.p, mp_, reg, diag_.p, st_);
      dense_cholesky<double>(ds64_, st_, &launches_);
      launches_ += 5;
      fp64_ready_ = true;
      if (stats_) stats_->factor_flops += (2.0 / 3.0) * std::pow(static_cast<double>(f_.n), 3.0);
    } else {
      launch_dense_clear<double>(M64_.p, order_, mp_, st_);
      launch_assemble<double>(amd_, x_.p, s_.p, qdiag_.p, free_.p, amode, reg, M64_.p, diag_.p, order_, mp_, st_);
      if (xspace_) launch_xspace_diag(dev_, mode == kWeightOnes ? 0 : 1, M64_.p, mp_, diag_.p, st_);
      dense_cholesky<double>(ds64_, st_, &launches_);
      launches_ += xspace_ ? 3 : 2;
      fp64_ready_ = true;
    }
  } else {
    launch_dense_clear<float>(M32_.p, f_.m, mp_, st_);
    launch_assemble<float>(amd_, x_.p, s_.p, qdiag_.p, free_.p, mode, reg, M32_.p, diag_.p, f_.m, mp_, st_);
    dense_cholesky_tc(ds32_, err_.p, st_, &launches_);
    launches_ += 2;
  }
  if (stats_) stats_->factor_flops += (2.0 / 3.0) * std::pow(static_cast<double>(order_), 3.0);
}

// Mehrotra's QP starting point (qp_interior_point.cpp:2891-2928), after the default start's system
// (the KKT without the Hessian: H = I, so M = A A') is factored and z holds its dy: xt = 1 + A'dy;
// (u, y) from the same system with r1 = -(c + Q xt), r2 = 0, i.e. A A' y = -A r1 and u = r1 + A'y;
// x and s = xt and -u shifted into the interior and balanced so that the products x_j s_j spread
// evenly; y = the least-squares dual.
void Engine::mehrotra_qp_start() {
  const int n = f_.n, m = f_.m;
  double* xt = dxa_.p;
  double* r1 = dsa_.p;
  double* w = ds_.p;
  launch_mehrotra_r1(dev_, xt, r1, st_);
  launch_rows_minus(dev_, r1, nullptr, st_);  // z = 0 - A r1
  newton_solve();                              // z = y_ls
  launch_add_atz(dev_, r1, w, st_);            // u = r1 + A'y_ls
  launches_ += 5;
  std::vector<double> hxt(n), hu(n), hy(m);
  std::vector<uint8_t> fr(f_.free_col.begin(), f_.free_col.end());
  SOV_CUDA(cudaMemcpyAsync(hxt.data(), xt, sizeof(double) * n, cudaMemcpyDeviceToHost, st_));
  SOV_CUDA(cudaMemcpyAsync(hu.data(), w, sizeof(double) * n, cudaMemcpyDeviceToHost, st_));
  if (m) SOV_CUDA(cudaMemcpyAsync(hy.data(), z_.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st_));
  SOV_CUDA(cudaStreamSynchronize(st_));
  double min_x = INFINITY, min_s = INFINITY;
  for (int j = 0; j < n; ++j) {
    if (fr[j]) continue;
    min_x = std::min(min_x, hxt[j]);
    min_s = std::min(min_s, -hu[j]);
  }
  const double shift_x = std::max(-1.5 * min_x, 0.0), shift_s = std::max(-1.5 * min_s, 0.0);
  double xs = 0.0, sum_x = 0.0, sum_s = 0.0;
  for (int j = 0; j < n; ++j) {
    if (fr[j]) continue;
    const double xh = hxt[j] + shift_x, sh = -hu[j] + shift_s;
    xs += xh * sh;
    sum_x += xh;
    sum_s += sh;
  }
  const double bal_x = sum_s > 0.0 ? 0.5 * xs / sum_s : 1.0;
  const double bal_s = sum_x > 0.0 ? 0.5 * xs / sum_x : 1.0;
  std::vector<double> hx(n), hs(n);
  for (int j = 0; j < n; ++j) {
    if (fr[j]) {
      hx[j] = hxt[j];
      hs[j] = 0.0;
      continue;
    }
    hx[j] = std::max(1e-8, hxt[j] + shift_x + bal_x);
    hs[j] = std::max(1e-8, -hu[j] + shift_s + bal_s);
  }
  x_.upload(hx.data(), n, st_);
  s_.upload(hs.data(), n, st_);
  if (m) y_.upload(hy.data(), m, st_);
}

// One Newton pass of a coupled-Hessian QP: z = rp - A H^-1 r1, M dy = z, dx = H^-1 (r1 + A'dy),
// then ds, the ratio tests and the step lengths as in the separable path.
void Engine::coupled_newton(int mode) {
  if (backend_ == kKkt) {
    // K [dx; -dy] = [r1; rp] in one refined solve
    if (stats_) stats_->solves++;
    launch_hessian_r1(dev_, mode, hvec_.p, st_);
    kkt_->solve_newton(hvec_.p, rp_.p, z_.p, st_, &launches_);
    launch_direction_dx(dev_, mode, hvec_.p, st_, &launches_);
    launches_ += 1;
    return;
  }
  launch_hessian_r1(dev_, mode, hvec_.p, st_);
  dense_solve<double>(dsh_, hvec_.p, epoch_, err_.p, st_, &launches_);
  launch_rows_minus(dev_, hvec_.p, rp_.p, st_);
  newton_solve();
  launch_hessian_w(dev_, mode, hvec_.p, st_);
  dense_solve<double>(dsh_, hvec_.p, epoch_, err_.p, st_, &launches_);
  launch_direction_dx(dev_, mode, hvec_.p, st_, &launches_);
  launches_ += 3;
}

bool Engine::newton_solve() {
  if (stats_) stats_->solves++;
  if (backend_ == kBand) {
    band_solve(bandsys_, z_.p, st_, &launches_);
    return true;
  }
  if (backend_ == kSparse) {
    sparse_.solve(z_.p, st_, &launches_);
    return true;
  }
  if (backend_ == kKkt) {
    kkt_->solve_normal(z_.p, st_, &launches_);
    return true;
  }
  if (backend_ == kDense64) {
    dense_solve<double>(ds64_, z_.p, epoch_, err_.p, st_, &launches_);
    return true;
  }
  // mixed: PCG on (A D A' + reg I) dy = z with the FP32 factor as preconditioner
  const int m = f_.m;
  const double reg = 1e-12;
  const double tol2 = 1e-22;  // ||r|| <= 1e-11 ||b||
  k_pcg_init<<<1, 1024, 0, st_>>>(m, z_.p, pcg_x_.p, pcg_r_.p, pcg_w_.p, pcg_s_.p);
  dense_solve<float>(ds32_, pcg_w_.p, epoch_, err_.p, st_, &launches_);
  k_pcg_direction<<<1, 1024, 0, st_>>>(m, pcg_r_.p, pcg_w_.p, pcg_p_.p, pcg_s_.p, 1);
  launches_ += 2;
  bool converged = false;
  const int cap = opt_.pcg_max_iterations > 0 ? opt_.pcg_max_iterations : 50;
  const int used_before = pcg_iterations_;
  for (int k = 0; k < cap; ++k) {
    launch_normal_matvec(dev_, pcg_p_.p, pcg_tmp_.p, pcg_q_.p, reg, st_);
    k_pcg_step<<<1, 1024, 0, st_>>>(m, pcg_p_.p, pcg_q_.p, pcg_x_.p, pcg_r_.p, pcg_w_.p, pcg_s_.p);
    SOV_CUDA(cudaMemcpyAsync(pcg_h_, pcg_s_.p, sizeof(PcgScalars), cudaMemcpyDeviceToHost, st_));
    SOV_CUDA(cudaStreamSynchronize(st_));
    launches_ += 3;
    ++pcg_iterations_;
    if (!(pcg_h_->rr > tol2 * pcg_h_->bb)) {
      converged = std::isfinite(pcg_h_->rr);
      break;
    }
    dense_solve<float>(ds32_, pcg_w_.p, epoch_, err_.p, st_, &launches_);
    k_pcg_direction<<<1, 1024, 0, st_>>>(m, pcg_r_.p, pcg_w_.p, pcg_p_.p, pcg_s_.p, 0);
    launches_ += 1;
  }
  if (!converged || pcg_iterations_ - used_before > kPcgSwitch) to_fp64_ = true;
  if (converged) {
    SOV_CUDA(cudaMemcpyAsync(z_.p, pcg_x_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, st_));
    return true;
  }
  // FP64 fallback for this iteration: factor in FP64 once, then solve directly
  if (!fp64_ready_) {
    ++fp64_fallbacks_;
    if (!M64_.p) {
      M64_.alloc(static_cast<size_t>(mp_) * mp_);
      Linv64_.alloc(static_cast<size_t>(nb_) * kNB * kNB);
      ds64_ = DenseSystem<double>{M64_.p, Linv64_.p, diag_.p, order_, mp_, nb_, &sc_.p->drops, &sc_.p->fail, flags_.p, flags_.p + nb_, 1e-13};
    }
    launch_dense_clear<double>(M64_.p, f_.m, mp_, st_);
    launch_assemble<double>(amd_, x_.p, s_.p, qdiag_.p, free_.p, last_mode_, reg, M64_.p, diag_.p, f_.m, mp_, st_);
    dense_cholesky<double>(ds64_, st_, &launches_);
    fp64_ready_ = true;
  }
  dense_solve<double>(ds64_, z_.p, epoch_, err_.p, st_, &launches_);
  return true;
}

void Engine::read_scalars() {
  SOV_CUDA(cudaMemcpyAsync(hs_.h, sc_.p, sizeof(IpmScalars), cudaMemcpyDeviceToHost, st_));
  SOV_CUDA(cudaStreamSynchronize(st_));
}

std::string Engine::describe() const {
  char buf[256];
  const char* space = xspace_ ? "x-space Q + A'ZW^-1A, " : "";
  if (backend_ == kKkt) {
    int len = std::snprintf(buf, sizeof buf,
                            "sparse quasi-definite LDL^T on the GPU with %s ordering (order %d, nnz(L) = %lld, %d levels)",
                            kkt_->ordering(), kkt_->order(), kkt_->nnz_l(), kkt_->levels());
    if (kkt_->delta() > 1e-9 && len > 0 && len < static_cast<int>(sizeof buf))
      std::snprintf(buf + len, sizeof buf - len, ", regularization raised to %g", kkt_->delta());
    return buf;
  }
  if (coupled_) {
    std::snprintf(buf, sizeof buf,
                  "A H^-1 A' with H = Q + X^-1 S dense, dense Cholesky on the GPU, FP64 (H %d x %d, %d x %d)", f_.n,
                  f_.n, order_, order_);
    return buf;
  }
  if (backend_ == kSparse)
    std::snprintf(buf, sizeof buf, "sparse LDL^T on the GPU with %s ordering (order %d, nnz(L) = %lld, %d levels)",
                  sym_.ordering == SparseOrder::kNestedDissection ? "nested-dissection" : "minimum-degree", order_,
                  sym_.nnz_l, sym_.levels());
  else if (backend_ == kBand)
    std::snprintf(buf, sizeof buf, "%sbanded LDL^T on the GPU (order %d, half-bandwidth %d)", space, order_, kd_);
  else if (backend_ == kDense64)
    std::snprintf(buf, sizeof buf, "%sdense Cholesky on the GPU, FP64 (%d x %d)%s", space, order_, order_,
                  sparse_refused_ ? "; the sparse factor would be nearly dense" : "");
  else
    std::snprintf(buf, sizeof buf,
                  "dense Cholesky on the GPU, FP32 preconditioned FP64 PCG (%d x %d, %d PCG iterations, %d FP64 "
                  "refactorizations)",
                  f_.m, f_.m, pcg_iterations_, fp64_fallbacks_);
  return buf;
}

void Engine::publish(const DevBuf<double>& x, const DevBuf<double>& y, const DevBuf<double>& s, int status,
                     int iteration, double gap, double pres, double dres, const std::string& msg, sov_result* r) {
  const int n = f_.n, m = f_.m;
  std::vector<double> hx(n), hy(m), hs(n);
  SOV_CUDA(cudaMemcpyAsync(hx.data(), x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st_));
  SOV_CUDA(cudaMemcpyAsync(hy.data(), y.p, sizeof(double) * m, cudaMemcpyDeviceToHost, st_));
  SOV_CUDA(cudaMemcpyAsync(hs.data(), s.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st_));
  SOV_CUDA(cudaStreamSynchronize(st_));
  r->status = status;
  r->iterations = iteration;
  r->duality_gap = gap;
  r->primal_residual = pres;
  r->dual_residual = dres;
  r->has_objective_value = 1;
  double obj = model_.obj_constant;
  if (!f_.qp) {
    // publish_iterate (interior_point.cpp:541-563)
    for (int j = 0; j < f_.n_struct; ++j) {
      const double v = f_.shift[j] + f_.col_scale[j] * hx[j];
      if (r->primal) r->primal[j] = v;
      if (r->dual_col) r->dual_col[j] = hs[j] / f_.col_scale[j];
      obj += (model_.obj ? model_.obj[j] : 0.0) * v;
    }
    if (r->dual_row)
      for (int i = 0; i < f_.m0; ++i) r->dual_row[i] = f_.row_scale[i] * hy[i];
  } else {
    // qp_interior_point.cpp:3018-3037 and capture_diagnostics (:2862-2877)
    std::vector<double> prim(f_.n_struct);
    for (int j = 0; j < f_.n_struct; ++j) prim[j] = f_.shift[j] + hx[j];
    for (int j = 0; j < f_.n_struct; ++j) obj += (model_.obj ? model_.obj[j] : 0.0) * prim[j];
    if (model_.q_col_ptr)
      for (int j = 0; j < f_.n_struct; ++j)
        for (int k = model_.q_col_ptr[j]; k < model_.q_col_ptr[j + 1]; ++k)
          obj += 0.5 * model_.q_values[k] * prim[model_.q_row_idx[k]] * prim[j];
    if (r->primal) std::copy(prim.begin(), prim.end(), r->primal);
    if (r->dual_col) std::copy(hs.begin(), hs.begin() + f_.n_struct, r->dual_col);
    if (r->dual_row) std::copy(hy.begin(), hy.begin() + f_.m0, r->dual_row);
  }
  if (captured_) {
    if (r->ipm_x) SOV_CUDA(cudaMemcpy(r->ipm_x, cx_.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
    if (r->ipm_y) SOV_CUDA(cudaMemcpy(r->ipm_y, cy_.p, sizeof(double) * m, cudaMemcpyDeviceToHost));
    if (r->ipm_s) SOV_CUDA(cudaMemcpy(r->ipm_s, cs_.p, sizeof(double) * n, cudaMemcpyDeviceToHost));
  } else {
    if (r->ipm_x) std::copy(hx.begin(), hx.end(), r->ipm_x);
    if (r->ipm_y) std::copy(hy.begin(), hy.end(), r->ipm_y);
    if (r->ipm_s) std::copy(hs.begin(), hs.end(), r->ipm_s);
  }
  r->objective_value = obj;
  std::snprintf(r->message, sizeof(r->message), "%s", msg.c_str());
}

void Engine::run(sov_result* r) {
  const int m = f_.m, n = f_.n;
  r->n_ipm = n;
  r->m_ipm = m;
  sov_diagnostics* dg = r->diagnostics;
  if (dg) {
    std::memset(dg, 0, sizeof(*dg));
    dg->scaling_applied = f_.scaling_applied;
    dg->coefficient_min_abs_before = f_.coef_min_before;
    dg->coefficient_max_abs_before = f_.coef_max_before;
    dg->coefficient_min_abs_after = f_.coef_min_after;
    dg->coefficient_max_abs_after = f_.coef_max_after;
    dg->stall_iteration = -1;
  }
  setup();
  cudaEvent_t e0, e1;
  SOV_CUDA(cudaEventCreate(&e0));
  SOV_CUDA(cudaEventCreate(&e1));
  SOV_CUDA(cudaEventRecord(e0, st_));

  // starting point (interior_point.cpp:488-506 / qp_interior_point.cpp:2881-2950, default start)
  auto default_start = [&]() {
    assemble_and_factor(kWeightOnes);
    if (xspace_) launch_start_rhs_x(dev_, st_, &launches_);
    else launch_start_rhs(dev_, st_, &launches_);
    dev_.start_system = 1;  // the mixed path's matrix-free operator weighs every column 1 as well
    newton_solve();
    if (xspace_) launch_start_dy_x(dev_, st_, &launches_);
    if (mehrotra_start_ && f_.qp && !xspace_ && f_.m > 0) {
      mehrotra_qp_start();
    } else {
      launch_start_point(dev_, st_, &launches_);
    }
    dev_.start_system = 0;
  };
  default_start();
  bool warm_used = false;
  if (opt_.warm_x && opt_.warm_y && opt_.warm_s) {
    // keep the supplied point when its residual metric beats the default start's
    launch_residuals(dev_, st_, &launches_);
    read_scalars();
    const double default_metric = hs_.h->metric, default_mu = hs_.h->mu;
    SOV_CUDA(cudaMemcpyAsync(bx_.p, x_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
    SOV_CUDA(cudaMemcpyAsync(bs_.p, s_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
    SOV_CUDA(cudaMemcpyAsync(by_.p, y_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, st_));
    x_.upload(opt_.warm_x, n, st_);
    y_.upload(opt_.warm_y, m, st_);
    s_.upload(opt_.warm_s, n, st_);
    launch_residuals(dev_, st_, &launches_);
    read_scalars();
    // safeguard against gross mispredictions: keep the supplied point unless its residual metric
    // is more than 10x the default start's (its mu is normally far smaller)
    if (std::isfinite(hs_.h->metric) && std::isfinite(hs_.h->mu) && hs_.h->metric <= 10.0 * default_metric &&
        hs_.h->mu <= default_mu) {
      warm_used = true;
    } else {
      SOV_CUDA(cudaMemcpyAsync(x_.p, bx_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(s_.p, bs_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(y_.p, by_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, st_));
    }
  }
  if (dg) dg->warm_start_used = warm_used ? 1 : 0;
  SOV_CUDA(cudaMemsetAsync(&sc_.p->fail, 0, sizeof(int), st_));

  SOV_CUDA(cudaMemcpyAsync(bx_.p, x_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
  SOV_CUDA(cudaMemcpyAsync(bs_.p, s_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
  SOV_CUDA(cudaMemcpyAsync(by_.p, y_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, st_));
  double best_metric = INFINITY, best_gap = INFINITY, best_p = INFINITY, best_d = INFINITY;
  int best_it = 0, stale = 0;
  bool done = false;
  std::string fail_msg;
  int it = 0;
  for (; it < opt_.max_iterations; ++it) {
    if (opt_.ipm_iterate_at == it + 1) {
      cx_.alloc(n);
      cy_.alloc(m);
      cs_.alloc(n);
      SOV_CUDA(cudaMemcpyAsync(cx_.p, x_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(cs_.p, s_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(cy_.p, y_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, st_));
      captured_ = true;
    }
    launch_residuals(dev_, st_, &launches_);
    read_scalars();
    const IpmScalars s = *hs_.h;
    if (it > 0) {
      const int prev = it - 1;
      const bool prev_sample = prev < 8 || prev % 10 == 0 || prev + 1 == opt_.max_iterations;
      if (dg && prev_sample && dg->step_history_len < SOV_HISTORY_MAX) {
        dg->primal_step_history[dg->step_history_len] = s.alpha_p;
        dg->dual_step_history[dg->step_history_len] = s.alpha_d;
        dg->step_history_len++;
      }
      if (dg && dg->stall_iteration == prev + 1) {
        dg->stall_primal_step = s.alpha_p;
        dg->stall_dual_step = s.alpha_d;
      }
    }
    if (s.fail || s.skipped) {
      fail_msg = f_.qp ? "QP-IPM Newton factorization failed."
                       : "IPM stopped because the affine predictor factorization failed; the best iterate is returned "
                         "with optimality unproven.";
      break;
    }
    if (s.metric < best_metric) {
      best_metric = s.metric;
      SOV_CUDA(cudaMemcpyAsync(bx_.p, x_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(bs_.p, s_.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, st_));
      SOV_CUDA(cudaMemcpyAsync(by_.p, y_.p, sizeof(double) * m, cudaMemcpyDeviceToDevice, st_));
      best_gap = s.gap;
      best_p = s.p_res;
      best_d = s.d_res;
      best_it = it + 1;
      stale = 0;
    } else {
      ++stale;
    }
    const bool sample = it < 8 || it % 10 == 0 || it + 1 == opt_.max_iterations;
    if (dg && sample && dg->history_len < SOV_HISTORY_MAX) {
      dg->history_iterations[dg->history_len] = it + 1;
      dg->objective_history[dg->history_len] = s.cx;
      dg->gap_history[dg->history_len] = s.gap;
      dg->mu_history[dg->history_len] = s.mu;
      dg->history_len++;
    }
    if (s.gap < best_gap) {
      best_gap = s.gap;
      stale = 0;
    } else if (stale >= 8 && dg && dg->stall_iteration < 0) {
      dg->stall_iteration = it + 1;
      dg->stall_gap = s.gap;
      dg->stall_mu = s.mu;
    }
    if (s.p_res < opt_.feasibility_tol && s.d_res < opt_.feasibility_tol && s.gap < opt_.optimality_tol) {
      SOV_CUDA(cudaEventRecord(e1, st_));
      const std::string msg =
          f_.qp ? "Optimal convex QP found by Mehrotra predictor-corrector IPM. KKT system: " +
                      std::string(backend_ == kKkt ? "" : "normal equations, ") + describe() + "."
                : "Optimal solution found by primal-dual interior-point (Mehrotra). Normal equations: " + describe() +
                      ".";
      publish(x_, y_, s_, SOV_OPTIMAL, it + 1, s.gap, s.p_res, s.d_res, msg, r);
      done = true;
      break;
    }
    // a supplied start that has not converged after kWarmGiveUp iterations is abandoned once: the
    // solve restarts from the default start (and so does its best-iterate record)
    if (warm_used && it + 1 == kWarmGiveUp) {
      warm_used = false;
      if (dg) dg->warm_start_used = 0;
      default_start();
      SOV_CUDA(cudaMemsetAsync(&sc_.p->fail, 0, sizeof(int), st_));
      best_metric = best_gap = best_p = best_d = INFINITY;
      best_it = 0;
      stale = 0;
      continue;
    }
    assemble_and_factor(f_.qp ? kWeightQp : kWeightLp);
    for (int pass : {kRhsAffine, kRhsCorrector}) {
      if (coupled_ || backend_ == kKkt) {
        coupled_newton(pass);
        continue;
      }
      if (xspace_) launch_newton_rhs_x(dev_, pass, st_, &launches_);
      else launch_newton_rhs(dev_, pass, st_, &launches_);
      newton_solve();
      if (xspace_) launch_direction_x(dev_, pass, st_, &launches_);
      else launch_direction(dev_, pass, st_, &launches_);
    }
    launch_update(dev_, st_, &launches_);
  }
  if (!done) SOV_CUDA(cudaEventRecord(e1, st_));
  SOV_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  SOV_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  r->solve_seconds = ms * 1e-3;
  int err_h = 0;
  SOV_CUDA(cudaMemcpy(&err_h, err_.p, sizeof(int), cudaMemcpyDeviceToHost));
  if (err_h) throw std::runtime_error("a dataflow triangular solve timed out waiting for a dependency");
  if (!done) {
    if (f_.qp) {
      // solve_qp_ipm failure exits publish the current point without an objective (:3042-3048, :3112-3115)
      const std::string msg = fail_msg.empty() ? "QP-IPM iteration limit reached without convergence." : fail_msg;
      publish(x_, y_, s_, SOV_ERROR, fail_msg.empty() ? it : best_it, best_gap, best_p, best_d, msg, r);
      r->has_objective_value = 0;
    } else {
      const int st = best_p <= opt_.feasibility_tol ? SOV_FEASIBLE : SOV_NUMERICAL_ERROR;
      std::string msg = fail_msg;
      if (msg.empty()) {
        char buf[512];
        std::snprintf(buf, sizeof buf,
                      "IPM stopped after %d iterations without meeting tolerance; returning best iterate from %d as "
                      "a lower-accuracy candidate. Relative duality gap = %g (tolerance %g), primal residual = %g, "
                      "dual residual = %g. Optimality is not proven.",
                      opt_.max_iterations, best_it, best_gap, opt_.optimality_tol, best_p, best_d);
        msg = buf;
      }
      publish(bx_, by_, bs_, st, best_it, best_gap, best_p, best_d, msg, r);
    }
  }
  if (dg) {
    dg->refactorizations = factorizations_;
    dg->pcg_iterations = pcg_iterations_;
    dg->fp64_fallbacks = fp64_fallbacks_;
  }
  if (stats_) {
    stats_->launches += launches_;
    stats_->factorizations += factorizations_;
    stats_->kernel_ms += ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (pcg_h_) g_pinned_slots.release(pcg_h_);
}

}  // namespace

int solve_single(const sov_model& model, const StdForm& f, const sov_options& opt, sov_result* result,
                 cudaStream_t stream, EngineStats* stats) {
  // separable QPs with free variables and narrow banded inequality rows (the convex-sequence
  // shape): the x-space double-double path; anything it does not bring to OPTIMAL under AUTO is
  // solved again by the general engine below
  if (f.qp && (opt.factorization == SOV_FACTOR_AUTO || opt.factorization == SOV_FACTOR_XSPACE)) {
    XBandModel xb;
    if (xband_prepare(model, &xb)) {
      solve_xband(model, xb, opt, result, stream, stats);
      if (result->status == SOV_OPTIMAL || opt.factorization == SOV_FACTOR_XSPACE) return SOV_OK;
    }
  }
  {
    Engine e(model, f, opt, stream, stats);
    e.run(result);
  }
  // QP: a second attempt from Mehrotra's starting point when the default start does not reach
  // OPTIMAL (qp_interior_point.cpp:3166-3180; SOVEREIGN_QP_DISABLE=retry turns it off, as there)
  if (!f.qp || result->status == SOV_OPTIMAL || f.m == 0 || opt.factorization == SOV_FACTOR_XSPACE) return SOV_OK;
  if (const char* off = std::getenv("SOVEREIGN_QP_DISABLE"))
    if ((std::string(",") + off + ",").find(",retry,") != std::string::npos) return SOV_OK;
  sov_result second = *result;
  std::vector<double> primal(f.n_struct), dual_col(f.n_struct), dual_row(f.m0), ix(f.n), iy(f.m), is(f.n);
  sov_diagnostics diag{};
  second.primal = result->primal ? primal.data() : nullptr;
  second.dual_col = result->dual_col ? dual_col.data() : nullptr;
  second.dual_row = result->dual_row ? dual_row.data() : nullptr;
  second.ipm_x = result->ipm_x ? ix.data() : nullptr;
  second.ipm_y = result->ipm_y ? iy.data() : nullptr;
  second.ipm_s = result->ipm_s ? is.data() : nullptr;
  second.diagnostics = result->diagnostics ? &diag : nullptr;
  {
    Engine e(model, f, opt, stream, stats, true);
    e.run(&second);
  }
  if (second.status == SOV_OPTIMAL) {
    auto put = [](double* dst, const std::vector<double>& src) {
      if (dst) std::copy(src.begin(), src.end(), dst);
    };
    put(result->primal, primal);
    put(result->dual_col, dual_col);
    put(result->dual_row, dual_row);
    put(result->ipm_x, ix);
    put(result->ipm_y, iy);
    put(result->ipm_s, is);
    if (result->diagnostics) *result->diagnostics = diag;
    const int first_iterations = result->iterations;
    sov_result keep = *result;  // the caller's array pointers
    *result = second;
    result->primal = keep.primal;
    result->dual_col = keep.dual_col;
    result->dual_row = keep.dual_row;
    result->ipm_x = keep.ipm_x;
    result->ipm_y = keep.ipm_y;
    result->ipm_s = keep.ipm_s;
    result->diagnostics = keep.diagnostics;
    result->iterations += first_iterations;
  } else {
    const std::string msg = std::string(result->message) + " | Mehrotra starting point: " + second.message;
    std::snprintf(result->message, sizeof(result->message), "%s", msg.c_str());
  }
  return SOV_OK;
}

}  // namespace sov
