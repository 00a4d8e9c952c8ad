// tc_chol.cu -- split-precision 3xTF32 tensor-core updates for the FP32 blocked Cholesky.
//
// The mixed-precision factor of A D A' (the preconditioner of the FP64 PCG) spends its flops in
// two products per 64-wide panel kb:
//   panel     L_ik = A_ik Linv_kk^T            (tiles of 128 rows x 64, K = 64)
//   trailing  A_ij -= L_ik L_jk^T, i >= j      (tiles of 128 x 128, K = 64)
// Both run on tcgen05 with FP32 accumulation in TMEM. Each FP32 operand a is split into
// a_hi = tf32(a) and a_lo = tf32(a - a_hi); the product keeps a_hi b_hi + a_hi b_lo + a_lo b_hi,
// three kind::tf32 MMAs into the same accumulator, which recovers close to FP32 accuracy.
// Operand layout in memory: column-major with leading dimension ld (element (r, k) at k*ld + r).
#include <algorithm>
#include <cstdlib>
#include <string>

#include "common.cuh"
#include "dense.cuh"
#include "gemm_ws.cuh"
#include "tc.cuh"

namespace sov {
namespace {

constexpr int kTcM = 128;       // MMA M (rows of a tile)
constexpr int kTcK = kNB;       // K of one panel (64)
constexpr int kTcThreads = 128; // 4 warps: one per 32 TMEM lanes

__device__ __forceinline__ float to_tf32(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

// One 128 x N tile: C(r, n) (+)= -sum_k A(r, k) B(n, k) with 3xTF32. rows/cols beyond `rows_valid`
// / `cols_valid` read as zero and are not stored.
template <int N>
__device__ void tc3_tile(float* C, int ldc, const float* A, int lda, const float* B, int ldb, int rows_valid,
                         int cols_valid, bool subtract, int* err) {
  extern __shared__ __align__(128) unsigned char smem[];
  constexpr int kABytes = kTcM * kTcK * 4;
  constexpr int kBBytes = N * kTcK * 4;
  unsigned char* a_hi = smem;
  unsigned char* a_lo = smem + kABytes;
  unsigned char* b_hi = smem + 2 * kABytes;
  unsigned char* b_lo = smem + 2 * kABytes + kBBytes;
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (warp == 0) tc::tmem_alloc(&tmem_base, N < 32 ? 32 : N);
  if (tid == 0) tc::mbar_init(&mbar, 1);
  // stage A and B: float4 loads along the contiguous row dimension, all of a thread's loads issued
  // before any use (operand origins and valid extents are multiples of 64 rows, so a float4 is
  // either wholly inside or wholly outside), then split into hi / lo in the K-major layout
  auto stage = [&](const float* src, int ld, int rows, int valid, unsigned char* hi_buf, unsigned char* lo_buf) {
    const int per_col = rows / 4;
    const int total = per_col * kTcK;
    constexpr int kMaxPer = (kTcM / 4) * kTcK / kTcThreads;  // 16
    float4 v[kMaxPer];
#pragma unroll
    for (int it = 0; it < kMaxPer; ++it) {
      const int idx = it * kTcThreads + tid;
      const int q = idx % per_col, k = idx / per_col;
      v[it] = (idx < total && 4 * q < valid)
                  ? __ldg(reinterpret_cast<const float4*>(src + static_cast<int64_t>(k) * ld + 4 * q))
                  : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int it = 0; it < kMaxPer; ++it) {
      const int idx = it * kTcThreads + tid;
      if (idx >= total) continue;
      const int q = idx % per_col, k = idx / per_col;
      const float e[4] = {v[it].x, v[it].y, v[it].z, v[it].w};
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const float h = to_tf32(e[u]);
        const uint32_t off = tc::kmajor_offset(4 * q + u, k, kTcK, 4);
        *reinterpret_cast<float*>(hi_buf + off) = h;
        *reinterpret_cast<float*>(lo_buf + off) = to_tf32(e[u] - h);
      }
    }
  };
  stage(A, lda, kTcM, rows_valid, a_hi, a_lo);
  stage(B, ldb, N, cols_valid, b_hi, b_lo);
  tc::fence_async_smem();
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  if (tid == 0) {
    constexpr uint32_t lbo = 128;                    // next 16-byte K chunk
    constexpr uint32_t sbo = (kTcK * 4 / 16) * 128;  // next group of 8 rows
    constexpr uint32_t idesc = tc::instr_desc(2, kTcM, N);
    const uint32_t ah = tc::smem_u32(a_hi), al = tc::smem_u32(a_lo);
    const uint32_t bh = tc::smem_u32(b_hi), bl = tc::smem_u32(b_lo);
#pragma unroll
    for (int s = 0; s < kTcK / 8; ++s) {  // K = 8 per tf32 MMA = two 16-byte chunks
      const uint32_t o = static_cast<uint32_t>(s) * 256;
      tc::mma<0>(tmem, tc::smem_desc(ah + o, lbo, sbo), tc::smem_desc(bh + o, lbo, sbo), idesc, s > 0);
      tc::mma<0>(tmem, tc::smem_desc(ah + o, lbo, sbo), tc::smem_desc(bl + o, lbo, sbo), idesc, 1);
      tc::mma<0>(tmem, tc::smem_desc(al + o, lbo, sbo), tc::smem_desc(bh + o, lbo, sbo), idesc, 1);
    }
    tc::commit(&mbar);
  }
  __syncwarp();
  const bool ok = tc::mbar_wait(&mbar, 0);
  if (!ok && lane == 0) atomicExch(err, 2);
  tc::fence_after();
  const int r = warp * 32 + lane;
  if (ok) {
#pragma unroll
    for (int cc = 0; cc < N / 32; ++cc) {
      float v[32];
      tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + cc * 32, v);
      if (r < rows_valid) {
#pragma unroll
        for (int c = 0; c < 32; ++c) {
          const int n = cc * 32 + c;
          if (n < cols_valid) {
            float* dst = C + static_cast<int64_t>(n) * ldc + r;
            *dst = subtract ? *dst - v[c] : v[c];
          }
        }
      }
    }
  } else {
    tc::mbar_wait(&mbar, 0);  // one more bounded wait for MMAs still in flight before freeing TMEM
  }
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, N < 32 ? 32 : N);
}

// Trailing update tiles of 128 x 128 over the lower trailing matrix after panel kb.
__global__ void __launch_bounds__(kTcThreads) k_tc3_syrk(float* M, int ld, int kb, int mp, int* err) {
  const int o = (kb + 1) * kNB;
  const int R = mp - o;
  int t = blockIdx.x, I = 0;
  while ((I + 1) * (I + 2) / 2 <= t) ++I;
  const int J = t - I * (I + 1) / 2;
  const int r0 = o + I * kTcM, c0 = o + J * kTcM;
  const float* A = M + static_cast<int64_t>(kb) * kNB * ld + r0;
  const float* B = M + static_cast<int64_t>(kb) * kNB * ld + c0;
  tc3_tile<kTcM>(M + static_cast<int64_t>(c0) * ld + r0, ld, A, ld, B, ld, min(kTcM + 0, mp - r0),
                 min(kTcM + 0, mp - c0), true, err);
  (void)R;
}

// Panel tiles: L_ik = A_ik Linv_kk^T for the rows below the diagonal block, 128 rows per CTA.
__global__ void __launch_bounds__(kTcThreads) k_tc3_trsm(float* M, int ld, int kb, int mp, const float* Linv,
                                                         int* err) {
  const int r0 = (kb + 1) * kNB + blockIdx.x * kTcM;
  float* panel = M + static_cast<int64_t>(kb) * kNB * ld + r0;
  // B(n, k) = Linv[n][k] = Lk[k * 64 + n]; the result overwrites the panel rows, so stage first:
  // tc3_tile reads all of A into shared memory before any store.
  tc3_tile<kNB>(panel, ld, panel, ld, Linv + static_cast<int64_t>(kb) * kNB * kNB, kNB, min(kTcM + 0, mp - r0), kNB,
                false, err);
}

}  // namespace

size_t tc3_smem_bytes(int N) { return static_cast<size_t>(2 * kTcM * kTcK * 4 + 2 * N * kTcK * 4); }

// FP32 blocked Cholesky with the panel and trailing products on the tensor cores: per 64-wide
// panel kb the diagonal block (FP32 factor and inverse), then the panel L_ik = A_ik Linv_kk^T and the
// trailing update A_ij -= L_ik L_jk^T on the lower tiles, both 3xTF32 products of the warp-specialised
// pipelined GEMM (gemm_ws.cuh). SOVEREIGN_TC_GEMM=single selects the single-stage tile kernels above.
void dense_cholesky_tc(const DenseSystem<float>& s, int* err, cudaStream_t st, int* launches) {
  static const bool single = [] {
    const char* e = std::getenv("SOVEREIGN_TC_GEMM");
    return e && std::string(e) == "single";
  }();
  once_per_device((const void*)k_tc3_syrk, [&] {
    SOV_CUDA(cudaFuncSetAttribute(k_tc3_syrk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc3_smem_bytes(kTcM)));
    SOV_CUDA(cudaFuncSetAttribute(k_tc3_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc3_smem_bytes(kNB)));
  });
  const long long ld = s.mp;
  int n = 0;
  for (int kb = 0; kb < s.nb; ++kb) {
    dense_potrf_block<float>(s, kb, st);
    ++n;
    const int o = (kb + 1) * kNB;
    const int rows = s.mp - o;
    if (rows > 0) {
      const int tiles = ceil_div(rows, kTcM);
      if (single) {
        k_tc3_trsm<<<tiles, kTcThreads, tc3_smem_bytes(kNB), st>>>(s.M, s.mp, kb, s.mp, s.Linv, err);
        k_tc3_syrk<<<tiles * (tiles + 1) / 2, kTcThreads, tc3_smem_bytes(kTcM), st>>>(s.M, s.mp, kb, s.mp, err);
      } else {
        float* panel = s.M + static_cast<long long>(kb) * kNB * ld + o;  // rows o.. of panel kb (column-major)
        // L_ik(r, n) = sum_k A_ik(r, k) Linv_kk(n, k); Linv_kk(n, k) sits at k * 64 + n
        WsGemmArgs t{panel, 1, ld, s.Linv + static_cast<long long>(kb) * kNB * kNB, 1, kNB, panel, 1, ld,
                     rows, kNB, kNB, 1.0f, 0.0f, nullptr, 0, err, 0};
        launch_gemm_ws<0>(t, st);
        // A_ij(r, c) -= sum_k L(r, k) L(c, k) on the trailing matrix's lower tiles
        WsGemmArgs u{panel, 1, ld, panel, 1, ld, s.M + o * ld + o, 1, ld, rows, rows, kNB, -1.0f, 1.0f, nullptr, 0,
                     err, 1};
        launch_gemm_ws<0>(u, st);
      }
      n += 2;
    }
  }
  SOV_LAUNCH_CHECK();
  if (launches) *launches += n;
}

}  // namespace sov
