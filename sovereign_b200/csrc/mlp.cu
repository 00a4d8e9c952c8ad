// mlp.cu -- the warm-start network: a small MLP trained and run with hand-written BF16 kernels.
//
// Network: n_in -> hidden x L (ReLU) -> n_out, FP32 master weights (Adam), BF16 operands in every
// product, FP32 accumulation. All three products of a layer run on one tcgen05 GEMM kernel,
//   forward     H' = act(H W^T + b)        A = H  (K-major),  B = W  (K-major)
//   input grad  dH = dH' W                  A = dH' (K-major), B = W^T (MN-major in memory)
//   weight grad dW = dH'^T H                A = dH'^T,         B = H^T (both MN-major in memory)
// whose loader reads FP32 operands with arbitrary strides, rounds them to BF16 and writes the
// canonical K-major shared-memory layout, so one kernel serves every transpose. The accumulator
// (128 x 128 FP32) lives in TMEM; the epilogue adds the bias, applies ReLU and scales.
// No counterpart in the reference (the warm start is new).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "batch.hpp"
#include "common.cuh"
#include "sov_ipm.h"
#include "gemm_ws.cuh"
#include "tc.cuh"

namespace sov {
namespace {

constexpr int kGM = 128, kGN = 128, kGK = 64, kGThreads = 128;

struct GemmArgs {
  const float* A;
  long long a_rs, a_ks;  // A(r, k) = A[r * a_rs + k * a_ks]
  const float* B;
  long long b_rs, b_ks;  // B(n, k) = B[n * b_rs + k * b_ks]
  float* C;
  long long c_rs, c_cs;  // C(r, n) = C[r * c_rs + n * c_cs]
  int M, N, K;
  float alpha, beta;     // C = alpha * A B^T + beta * C
  const float* bias;     // per column n (or null)
  int relu;
  int* err;
};

// C (M x N) = alpha A B^T + beta C (+ bias, ReLU), BF16 operands, FP32 accumulate in TMEM.
__global__ void __launch_bounds__(kGThreads) k_gemm_bf16(GemmArgs g) {
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* sa = smem;
  unsigned char* sb = smem + kGM * kGK * 2;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = blockIdx.y * kGM, n0 = blockIdx.x * kGN;
  if (warp == 0) tc::tmem_alloc(&tmem_base, kGN);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = tc::instr_desc(1, kGM, kGN);  // BF16 x BF16 -> FP32
  constexpr uint32_t lbo = 128, sbo = (kGK * 2 / 16) * 128;
  bool ok = true;
  uint32_t phase = 0;
  const int nk = (g.K + kGK - 1) / kGK;
  for (int kc = 0; kc < nk; ++kc) {
    const int k0 = kc * kGK;
    // stage A and B (iterate the contiguous dimension fastest)
    for (int idx = tid; idx < kGM * kGK; idx += kGThreads) {
      int r, k;
      if (g.a_ks == 1) {
        r = idx / kGK;
        k = idx % kGK;
      } else {
        k = idx / kGM;
        r = idx % kGM;
      }
      const int gr = r0 + r, gk = k0 + k;
      const float v = (gr < g.M && gk < g.K) ? g.A[gr * g.a_rs + gk * g.a_ks] : 0.0f;
      *reinterpret_cast<__nv_bfloat16*>(sa + tc::kmajor_offset(r, k, kGK, 2)) = __float2bfloat16_rn(v);
    }
    for (int idx = tid; idx < kGN * kGK; idx += kGThreads) {
      int n, k;
      if (g.b_ks == 1) {
        n = idx / kGK;
        k = idx % kGK;
      } else {
        k = idx / kGN;
        n = idx % kGN;
      }
      const int gn = n0 + n, gk = k0 + k;
      const float v = (gn < g.N && gk < g.K) ? g.B[gn * g.b_rs + gk * g.b_ks] : 0.0f;
      *reinterpret_cast<__nv_bfloat16*>(sb + tc::kmajor_offset(n, k, kGK, 2)) = __float2bfloat16_rn(v);
    }
    tc::fence_async_smem();
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (tid == 0) {
      const uint32_t a = tc::smem_u32(sa), b = tc::smem_u32(sb);
#pragma unroll
      for (int s = 0; s < kGK / 16; ++s) {  // K = 16 per BF16 MMA = two 16-byte chunks
        const uint32_t o = static_cast<uint32_t>(s) * 256;
        tc::mma<1>(tmem, tc::smem_desc(a + o, lbo, sbo), tc::smem_desc(b + o, lbo, sbo), idesc, (kc > 0 || s > 0));
      }
      tc::commit(&mbar);
    }
    __syncwarp();
    // the next chunk overwrites shared memory: wait for this chunk's MMAs
    if (!tc::mbar_wait(&mbar, phase)) {
      ok = false;
      if (lane == 0) atomicExch(g.err, 3);
    }
    phase ^= 1;
    tc::fence_after();
    __syncthreads();
    if (!ok) break;
  }
  if (ok) {
    const int r = r0 + warp * 32 + lane;
#pragma unroll 1
    for (int cc = 0; cc < kGN / 32; ++cc) {
      float v[32];
      tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + cc * 32, v);
      if (r < g.M) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int n = n0 + cc * 32 + c;
          if (n >= g.N) continue;
          float* dst = g.C + r * g.c_rs + n * g.c_cs;
          float out = g.alpha * (nk > 0 ? v[c] : 0.0f);
          if (g.beta != 0.0f) out += g.beta * *dst;
          if (g.bias) out += g.bias[n];
          if (g.relu) out = fmaxf(out, 0.0f);
          *dst = out;
        }
      }
    }
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kGN);
}

// Every product of the network: the warp-specialised multi-stage tcgen05 GEMM (gemm_ws.cuh), BF16
// operands, FP32 accumulation. SOVEREIGN_MLP_GEMM=single selects the single-stage kernel above.
void gemm(const GemmArgs& g, cudaStream_t st) {
  static const bool single = [] {
    const char* e = std::getenv("SOVEREIGN_MLP_GEMM");
    return e && std::string(e) == "single";
  }();
  if (!single) {
    WsGemmArgs w{g.A, g.a_rs, g.a_ks, g.B, g.b_rs, g.b_ks, g.C, g.c_rs, g.c_cs, g.M, g.N, g.K,
                 g.alpha, g.beta, g.bias, g.relu, g.err, 0};
    launch_gemm_ws<1>(w, st);
    return;
  }
  const size_t smem = static_cast<size_t>(kGM + kGN) * kGK * 2;
  once_per_device((const void*)k_gemm_bf16, [&] {
    SOV_CUDA(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  });
  dim3 grid(ceil_div(g.N, kGN), ceil_div(g.M, kGM));
  k_gemm_bf16<<<grid, kGThreads, smem, st>>>(g);
  SOV_LAUNCH_CHECK();
}

// ---- elementwise kernels ----
__global__ void k_relu_backward(float* dh, const float* h, long long count) {
  for (long long i = blockIdx.x * 256ll + threadIdx.x; i < count; i += gridDim.x * 256ll)
    if (h[i] <= 0.0f) dh[i] = 0.0f;
}

// dY = (Y - T) * 2 / (B * n_out); per-block partial loss sums (FP64)
__global__ void k_mse_grad(const float* y, const float* t, float* dy, long long count, float scale, double* part) {
  __shared__ double red[256];
  double acc = 0.0;
  for (long long i = blockIdx.x * 256ll + threadIdx.x; i < count; i += gridDim.x * 256ll) {
    const float d = y[i] - t[i];
    dy[i] = 2.0f * d * scale;
    acc += static_cast<double>(d) * d;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// db[n] = sum_b dH[b][n]
__global__ void k_colsum(const float* dh, int B, int N, float* db) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float acc = 0.0f;
  for (int b = 0; b < B; ++b) acc += dh[static_cast<long long>(b) * N + n];
  db[n] = acc;
}

__global__ void k_adam(float* w, const float* g, float* m, float* v, long long count, float lr, float b1, float b2,
                       float c1, float c2, float eps) {
  for (long long i = blockIdx.x * 256ll + threadIdx.x; i < count; i += gridDim.x * 256ll) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

__global__ void k_gather_rows(const float* src, const int* idx, int rows, int cols, float* dst) {
  const long long total = static_cast<long long>(rows) * cols;
  for (long long i = blockIdx.x * 256ll + threadIdx.x; i < total; i += gridDim.x * 256ll) {
    const int r = static_cast<int>(i / cols), c = static_cast<int>(i % cols);
    dst[i] = src[static_cast<long long>(idx[r]) * cols + c];
  }
}

// network input from raw parameters: (p - mean) / std in FP64, rounded to FP32
__global__ void k_normalize_in(const double* __restrict__ p, const double* __restrict__ mean,
                               const double* __restrict__ sd, long long count, int cols, float* __restrict__ out) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int c = static_cast<int>(i % cols);
    out[i] = static_cast<float>((p[i] - mean[c]) / sd[c]);
  }
}

// warm start from the network output o (log x, y, log s normalized): v = o * std + mean in FP64,
// x = max(exp(clip(v, -40, 40)), delta) on the first n columns, y = v on the next m, s like x on
// the last n; written as three row-major arrays
__global__ void k_decode_start(const float* __restrict__ o, const double* __restrict__ mean,
                               const double* __restrict__ sd, long long rows, int n, int m, double delta,
                               double* __restrict__ x, double* __restrict__ y, double* __restrict__ s) {
  const int cols = 2 * n + m;
  const long long count = rows * cols;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < count;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long r = i / cols;
    const int c = static_cast<int>(i % cols);
    const double v = static_cast<double>(o[i]) * sd[c] + mean[c];
    if (c < n) {
      x[r * n + c] = fmax(exp(fmin(fmax(v, -40.0), 40.0)), delta);
    } else if (c < n + m) {
      y[r * m + (c - n)] = v;
    } else {
      s[r * n + (c - n - m)] = fmax(exp(fmin(fmax(v, -40.0), 40.0)), delta);
    }
  }
}

template <class T>
struct Buf {
  T* p = nullptr;
  size_t n = 0;
  void alloc(size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    n = count;
    if (count) SOV_CUDA(cudaMalloc(&p, sizeof(T) * count));
  }
  ~Buf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

struct Mlp {
  std::vector<int> dims;  // n_in, h..., n_out
  std::vector<long long> w_off, b_off;
  long long nparam = 0;
  Buf<float> params, grads, adam_m, adam_v;
  int batch_cap = 0;
  std::vector<Buf<float>> act;   // act[0] = X, act[l+1] = output of layer l
  std::vector<Buf<float>> dact;  // gradients of the activations
  Buf<float> target;
  Buf<double> part;
  Buf<double> raw_in, norm, start;  // warm-start prediction: parameters, normalizers, decoded start
  // pinned landing buffer of the decoded starts (grow-only): the D2H runs at full speed, and the
  // caller's (pageable) arrays are filled from it on several threads
  struct Pinned {
    void* p = nullptr;
    size_t cap = 0;
    void* get(size_t bytes) {
      if (bytes > cap) {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
        SOV_CUDA(cudaMallocHost(&p, bytes));
        cap = bytes;
      }
      return p;
    }
    ~Pinned() {
      if (p) cudaFreeHost(p);
    }
  } landing, staging;  // the decoded starts out; the parameters in
  cudaEvent_t predicted = nullptr;  // starts written (sov_lp_solve_batch_predicted)
  Buf<int> err;
  long long step = 0;
  cudaStream_t st = nullptr;

  int layers() const { return static_cast<int>(dims.size()) - 1; }
  float* W(int l) { return params.p + w_off[l]; }
  float* bvec(int l) { return params.p + b_off[l]; }
  float* dW(int l) { return grads.p + w_off[l]; }
  float* db(int l) { return grads.p + b_off[l]; }

  void ensure_batch(int B) {
    if (B <= batch_cap) return;
    act.resize(dims.size());
    dact.resize(dims.size());
    for (size_t l = 0; l < dims.size(); ++l) {
      act[l].alloc(static_cast<size_t>(B) * dims[l]);
      dact[l].alloc(static_cast<size_t>(B) * dims[l]);
    }
    target.alloc(static_cast<size_t>(B) * dims.back());
    batch_cap = B;
  }

  void forward(int B) {
    for (int l = 0; l < layers(); ++l) {
      GemmArgs g{act[l].p, dims[l], 1, W(l), dims[l], 1, act[l + 1].p, dims[l + 1], 1,
                 B, dims[l + 1], dims[l], 1.0f, 0.0f, bvec(l), l + 1 < layers(), err.p};
      gemm(g, st);
    }
  }

  double loss_and_backward(int B) {
    const int L = layers();
    const long long cnt = static_cast<long long>(B) * dims[L];
    const int blocks = std::min<long long>(1184, (cnt + 255) / 256);
    k_mse_grad<<<blocks, 256, 0, st>>>(act[L].p, target.p, dact[L].p, cnt, 1.0f / static_cast<float>(cnt), part.p);
    for (int l = L - 1; l >= 0; --l) {
      // dW_l = dA_{l+1}^T A_l : (d_out x B) (B x d_in)
      GemmArgs gw{dact[l + 1].p, 1, dims[l + 1], act[l].p, 1, dims[l], dW(l), dims[l], 1,
                  dims[l + 1], dims[l], B, 1.0f, 0.0f, nullptr, 0, err.p};
      gemm(gw, st);
      k_colsum<<<ceil_div(dims[l + 1], 256), 256, 0, st>>>(dact[l + 1].p, B, dims[l + 1], db(l));
      if (l > 0) {
        // dA_l = dA_{l+1} W_l : (B x d_out)(d_out x d_in), then the ReLU mask of A_l
        GemmArgs gx{dact[l + 1].p, dims[l + 1], 1, W(l), 1, dims[l], dact[l].p, dims[l], 1,
                    B, dims[l], dims[l + 1], 1.0f, 0.0f, nullptr, 0, err.p};
        gemm(gx, st);
        const long long c2 = static_cast<long long>(B) * dims[l];
        k_relu_backward<<<std::min<long long>(1184, (c2 + 255) / 256), 256, 0, st>>>(dact[l].p, act[l].p, c2);
      }
    }
    SOV_LAUNCH_CHECK();
    std::vector<double> h(blocks);
    SOV_CUDA(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * blocks, cudaMemcpyDeviceToHost, st));
    SOV_CUDA(cudaStreamSynchronize(st));
    int e = 0;
    SOV_CUDA(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) throw CudaError("tensor-core GEMM wait ran out");
    return std::accumulate(h.begin(), h.end(), 0.0) / static_cast<double>(cnt);
  }

  void adam(float lr) {
    ++step;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(step)), c2 = 1.0f - std::pow(b2, static_cast<float>(step));
    k_adam<<<std::min<long long>(1184, (nparam + 255) / 256), 256, 0, st>>>(params.p, grads.p, adam_m.p, adam_v.p,
                                                                           nparam, lr, b1, b2, c1, c2, 1e-8f);
    SOV_LAUNCH_CHECK();
  }
};

}  // namespace sov

using sov::Mlp;

extern "C" {

int sov_mlp_create(int32_t n_in, int32_t hidden, int32_t hidden_layers, int32_t n_out, uint64_t seed, sov_mlp** out) {
  if (n_in <= 0 || hidden <= 0 || hidden_layers < 0 || n_out <= 0 || !out) return SOV_E_ARGUMENT;
  try {
    auto m = new Mlp();
    m->dims.push_back(n_in);
    for (int l = 0; l < hidden_layers; ++l) m->dims.push_back(hidden);
    m->dims.push_back(n_out);
    long long off = 0;
    for (int l = 0; l < m->layers(); ++l) {
      m->w_off.push_back(off);
      off += static_cast<long long>(m->dims[l + 1]) * m->dims[l];
      m->b_off.push_back(off);
      off += m->dims[l + 1];
    }
    m->nparam = off;
    // He-uniform initialisation from the seed
    std::vector<float> h(off, 0.0f);
    std::mt19937_64 rng(seed);
    for (int l = 0; l < m->layers(); ++l) {
      const float a = std::sqrt(6.0f / static_cast<float>(m->dims[l]));
      std::uniform_real_distribution<float> U(-a, a);
      for (long long k = 0; k < static_cast<long long>(m->dims[l + 1]) * m->dims[l]; ++k) h[m->w_off[l] + k] = U(rng);
    }
    m->params.alloc(off);
    m->grads.alloc(off);
    m->adam_m.alloc(off);
    m->adam_v.alloc(off);
    SOV_CUDA(cudaMemcpy(m->params.p, h.data(), sizeof(float) * off, cudaMemcpyHostToDevice));
    SOV_CUDA(cudaMemset(m->adam_m.p, 0, sizeof(float) * off));
    SOV_CUDA(cudaMemset(m->adam_v.p, 0, sizeof(float) * off));
    m->part.alloc(1184);
    m->err.alloc(1);
    SOV_CUDA(cudaMemset(m->err.p, 0, sizeof(int)));
    SOV_CUDA(cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking));
    *out = reinterpret_cast<sov_mlp*>(m);
    return SOV_OK;
  } catch (const std::exception&) {
    return SOV_E_CUDA;
  }
}

int64_t sov_mlp_param_count(const sov_mlp* h) { return h ? reinterpret_cast<const Mlp*>(h)->nparam : -1; }

int sov_mlp_get_params(const sov_mlp* h, float* params, int64_t count) {
  auto m = reinterpret_cast<const Mlp*>(h);
  if (!m || !params || count != m->nparam) return SOV_E_ARGUMENT;
  return cudaMemcpy(params, m->params.p, sizeof(float) * count, cudaMemcpyDeviceToHost) == cudaSuccess ? SOV_OK
                                                                                                       : SOV_E_CUDA;
}

int sov_mlp_set_params(sov_mlp* h, const float* params, int64_t count) {
  auto m = reinterpret_cast<Mlp*>(h);
  if (!m || !params || count != m->nparam) return SOV_E_ARGUMENT;
  return cudaMemcpy(m->params.p, params, sizeof(float) * count, cudaMemcpyHostToDevice) == cudaSuccess ? SOV_OK
                                                                                                       : SOV_E_CUDA;
}

int sov_mlp_forward(sov_mlp* h, const float* x, int32_t batch, float* y) {
  auto m = reinterpret_cast<Mlp*>(h);
  if (!m || !x || !y || batch <= 0) return SOV_E_ARGUMENT;
  try {
    m->ensure_batch(batch);
    SOV_CUDA(cudaMemcpyAsync(m->act[0].p, x, sizeof(float) * batch * m->dims[0], cudaMemcpyHostToDevice, m->st));
    m->forward(batch);
    SOV_CUDA(cudaMemcpyAsync(y, m->act.back().p, sizeof(float) * batch * m->dims.back(), cudaMemcpyDeviceToHost,
                             m->st));
    SOV_CUDA(cudaStreamSynchronize(m->st));
    return SOV_OK;
  } catch (const std::exception&) {
    return SOV_E_CUDA;
  }
}

namespace {

// Normalization, the network and the decoding of `batch` starts on the device: returns the decoded
// [x (batch*n_ipm) | y (batch*m_ipm) | s (batch*n_ipm)] in m->start, stream m->st (not synchronized).
double* predict_on_device(Mlp* m, const double* params, int batch, const double* in_mean, const double* in_std,
                          const double* out_mean, const double* out_std, int n_ipm, int m_ipm, double delta) {
  const int n_in = m->dims[0], n_out = m->dims.back();
  m->ensure_batch(batch);
  const size_t cnt_in = static_cast<size_t>(batch) * n_in, cnt_out = static_cast<size_t>(batch) * n_out;
  if (m->raw_in.n < cnt_in) m->raw_in.alloc(cnt_in);
  if (m->norm.n < static_cast<size_t>(2 * (n_in + n_out))) m->norm.alloc(2 * (n_in + n_out));
  if (m->start.n < cnt_out) m->start.alloc(cnt_out);
  double* nm = m->norm.p;
  double* hs = static_cast<double*>(m->staging.get(sizeof(double) * cnt_in));
  sov::parallel_memcpy(hs, params, sizeof(double) * cnt_in);
  SOV_CUDA(cudaMemcpyAsync(m->raw_in.p, hs, sizeof(double) * cnt_in, cudaMemcpyHostToDevice, m->st));
  SOV_CUDA(cudaMemcpyAsync(nm, in_mean, sizeof(double) * n_in, cudaMemcpyHostToDevice, m->st));
  SOV_CUDA(cudaMemcpyAsync(nm + n_in, in_std, sizeof(double) * n_in, cudaMemcpyHostToDevice, m->st));
  SOV_CUDA(cudaMemcpyAsync(nm + 2 * n_in, out_mean, sizeof(double) * n_out, cudaMemcpyHostToDevice, m->st));
  SOV_CUDA(cudaMemcpyAsync(nm + 2 * n_in + n_out, out_std, sizeof(double) * n_out, cudaMemcpyHostToDevice, m->st));
  sov::k_normalize_in<<<1184, 256, 0, m->st>>>(m->raw_in.p, nm, nm + n_in, static_cast<long long>(cnt_in), n_in,
                                              m->act[0].p);
  m->forward(batch);
  double* dx = m->start.p;
  double* dy = dx + static_cast<size_t>(batch) * n_ipm;
  double* ds = dy + static_cast<size_t>(batch) * m_ipm;
  sov::k_decode_start<<<1184, 256, 0, m->st>>>(m->act.back().p, nm + 2 * n_in, nm + 2 * n_in + n_out, batch, n_ipm,
                                              m_ipm, delta, dx, dy, ds);
  SOV_CUDA(cudaGetLastError());
  return dx;
}

}  // namespace

int sov_mlp_predict_start(sov_mlp* h, const double* params, int32_t batch, const double* in_mean,
                          const double* in_std, const double* out_mean, const double* out_std, int32_t n_ipm,
                          int32_t m_ipm, double delta, double* x, double* y, double* s) {
  auto m = reinterpret_cast<Mlp*>(h);
  if (!m || !params || !in_mean || !in_std || !out_mean || !out_std || !x || !y || !s || batch <= 0 || n_ipm < 0 ||
      m_ipm < 0 || 2 * n_ipm + m_ipm != m->dims.back())
    return SOV_E_ARGUMENT;
  try {
    double* dx = predict_on_device(m, params, batch, in_mean, in_std, out_mean, out_std, n_ipm, m_ipm, delta);
    // [x | y | s] are adjacent on the device: one copy into the pinned landing buffer
    const size_t cnt_out = static_cast<size_t>(batch) * m->dims.back();
    double* hl = static_cast<double*>(m->landing.get(sizeof(double) * cnt_out));
    SOV_CUDA(cudaMemcpyAsync(hl, dx, sizeof(double) * cnt_out, cudaMemcpyDeviceToHost, m->st));
    SOV_CUDA(cudaStreamSynchronize(m->st));
    const size_t nx = static_cast<size_t>(batch) * n_ipm, ny = static_cast<size_t>(batch) * m_ipm;
    sov::parallel_memcpy(x, hl, sizeof(double) * nx);
    sov::parallel_memcpy(y, hl + nx, sizeof(double) * ny);
    sov::parallel_memcpy(s, hl + nx + ny, sizeof(double) * nx);
    return SOV_OK;
  } catch (const std::exception&) {
    return SOV_E_CUDA;
  }
}

int sov_lp_solve_batch_predicted(sov_mlp* h, const double* params, const double* in_mean, const double* in_std,
                                 const double* out_mean, const double* out_std, int32_t n_ipm, int32_t m_ipm,
                                 double delta, int32_t count, const sov_model* models, const sov_options* opt,
                                 sov_result* results) {
  auto m = reinterpret_cast<Mlp*>(h);
  if (!m || !params || !in_mean || !in_std || !out_mean || !out_std || !models || !results || count <= 0 ||
      n_ipm < 0 || m_ipm < 0 || 2 * n_ipm + m_ipm != m->dims.back())
    return SOV_E_ARGUMENT;
  try {
    // the prediction runs on the network's stream while the host builds the first part; each part
    // gathers its starts after the event
    double* dx = predict_on_device(m, params, count, in_mean, in_std, out_mean, out_std, n_ipm, m_ipm, delta);
    if (!m->predicted) SOV_CUDA(cudaEventCreateWithFlags(&m->predicted, cudaEventDisableTiming));
    SOV_CUDA(cudaEventRecord(m->predicted, m->st));
    const sov::DeviceStarts st{dx, dx + static_cast<size_t>(count) * n_ipm,
                               dx + static_cast<size_t>(count) * (n_ipm + m_ipm), n_ipm, m_ipm, m->predicted};
    const int rc = sov::solve_batch(count, models, opt, 0, results, &st);
    SOV_CUDA(cudaStreamSynchronize(m->st));
    return rc;
  } catch (const sov::CudaError&) {
    cudaStreamSynchronize(m->st);  // the pinned input staging is reused by the next call
    return SOV_E_CUDA;
  } catch (const std::exception&) {
    cudaStreamSynchronize(m->st);
    return SOV_E_ARGUMENT;
  }
}

int sov_mlp_loss_grad(sov_mlp* h, const float* x, const float* t, int32_t batch, double* loss, float* grad) {
  auto m = reinterpret_cast<Mlp*>(h);
  if (!m || !x || !t || batch <= 0) return SOV_E_ARGUMENT;
  try {
    m->ensure_batch(batch);
    SOV_CUDA(cudaMemcpyAsync(m->act[0].p, x, sizeof(float) * batch * m->dims[0], cudaMemcpyHostToDevice, m->st));
    SOV_CUDA(cudaMemcpyAsync(m->target.p, t, sizeof(float) * batch * m->dims.back(), cudaMemcpyHostToDevice, m->st));
    m->forward(batch);
    const double l = m->loss_and_backward(batch);
    if (loss) *loss = l;
    if (grad) SOV_CUDA(cudaMemcpy(grad, m->grads.p, sizeof(float) * m->nparam, cudaMemcpyDeviceToHost));
    return SOV_OK;
  } catch (const std::exception&) {
    return SOV_E_CUDA;
  }
}

int sov_mlp_train(sov_mlp* h, const float* x, const float* t, int32_t count, int32_t epochs, int32_t batch,
                  float lr, uint64_t seed, double* final_loss) {
  auto m = reinterpret_cast<Mlp*>(h);
  if (!m || !x || !t || count <= 0 || epochs <= 0 || batch <= 0) return SOV_E_ARGUMENT;
  try {
    const int B = std::min(batch, count);
    m->ensure_batch(B);
    const int n_in = m->dims.front(), n_out = m->dims.back();
    sov::Buf<float> X, T;
    sov::Buf<int> idx;
    X.alloc(static_cast<size_t>(count) * n_in);
    T.alloc(static_cast<size_t>(count) * n_out);
    idx.alloc(count);
    SOV_CUDA(cudaMemcpy(X.p, x, sizeof(float) * count * n_in, cudaMemcpyHostToDevice));
    SOV_CUDA(cudaMemcpy(T.p, t, sizeof(float) * count * n_out, cudaMemcpyHostToDevice));
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::mt19937_64 rng(seed);
    double last = 0.0;
    for (int e = 0; e < epochs; ++e) {
      std::shuffle(order.begin(), order.end(), rng);
      SOV_CUDA(cudaMemcpy(idx.p, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice));
      double sum = 0.0;
      int nb = 0;
      for (int b0 = 0; b0 + B <= count; b0 += B) {
        sov::k_gather_rows<<<1184, 256, 0, m->st>>>(X.p, idx.p + b0, B, n_in, m->act[0].p);
        sov::k_gather_rows<<<1184, 256, 0, m->st>>>(T.p, idx.p + b0, B, n_out, m->target.p);
        m->forward(B);
        sum += m->loss_and_backward(B);
        m->adam(lr);
        ++nb;
      }
      last = nb ? sum / nb : 0.0;
    }
    SOV_CUDA(cudaStreamSynchronize(m->st));
    if (final_loss) *final_loss = last;
    return SOV_OK;
  } catch (const std::exception&) {
    return SOV_E_CUDA;
  }
}

void sov_mlp_destroy(sov_mlp* h) {
  auto m = reinterpret_cast<Mlp*>(h);
  if (!m) return;
  if (m->st) cudaStreamDestroy(m->st);
  if (m->predicted) cudaEventDestroy(m->predicted);
  delete m;
}

}  // extern "C"
