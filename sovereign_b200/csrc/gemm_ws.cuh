// gemm_ws.cuh -- warp-specialised tcgen05 GEMM with a multi-stage shared-memory ring.
//
//   C(r, n) = alpha * sum_k A(r, k) B(n, k) + beta * C(r, n) (+ bias[n], ReLU)
//
// One 128 x 128 output tile per CTA (all tiles, or those on or below the diagonal). Operands are FP32 in global
// memory with arbitrary row / K strides; they stream through kStages shared-memory stages in K
// chunks. Warps 0-3 are producers: each thread converts its 16-byte groups of a chunk (coalesced
// along whichever operand dimension is contiguous) to the tensor-core type and stores them in the
// canonical K-major no-swizzle layout (8-row x 16-byte core matrices; LBO 128 B, SBO 1024 B), then
// arrives on the stage's "full" barrier. Lane 0 of warp 4 issues tcgen05.mma from the stage into a
// TMEM accumulator (128 lanes x 128 FP32 columns) and commits the stage's "empty" barrier, so
// loading chunk k + kStages - 1 overlaps the MMAs of chunk k. After the last chunk the MMA thread
// commits "done" and warps 0-3 read the accumulator back with tcgen05.ld for the epilogue.
//   KIND 1: BF16 operands (kind::f16, K = 16 per MMA), 64-wide K chunks, 4 stages (128 KB).
//   KIND 0: 3xTF32 (kind::tf32, K = 8 per MMA): each FP32 operand split into hi = tf32(a) and
//           lo = tf32(a - hi); a_hi b_hi + a_hi b_lo + a_lo b_hi accumulate in FP32, close to FP32
//           products; 32-wide K chunks, 3 stages of four operand tiles (192 KB).
// Every barrier wait is bounded; a wait that runs out sets *err and the CTA winds down without
// touching C (it still waits, bounded, for MMAs in flight before releasing TMEM).
#pragma once

#include <cuda_bf16.h>

#include <cstdint>

#include "common.cuh"
#include "tc.cuh"

namespace sov {

struct WsGemmArgs {
  const float* A;
  long long a_rs, a_ks;  // A(r, k) = A[r * a_rs + k * a_ks]
  const float* B;
  long long b_rs, b_ks;  // B(n, k) = B[n * b_rs + k * b_ks]
  float* C;
  long long c_rs, c_cs;  // C(r, n) = C[r * c_rs + n * c_cs]
  int M, N, K;
  float alpha, beta;
  const float* bias;     // per column n, or null
  int relu;
  int* err;
  int lower;             // 1: only the tiles on or below the diagonal (I >= J), one CTA each
};

namespace wsg {

constexpr int kTile = 128;
constexpr int kThreads = 160;       // warps 0-3: producers and epilogue; warp 4: MMA issue
constexpr int kOperandBytes = 16384;  // 128 rows x 128 bytes of K
constexpr long long kWaitLimit = 1ll << 22;  // try_wait polls: a few seconds at most

template <int KIND>
struct Cfg;
template <>
struct Cfg<1> {  // BF16
  static constexpr int kK = 64, kStages = 4, kOperands = 2, kGroup = 8;
};
template <>
struct Cfg<0> {  // 3xTF32
  static constexpr int kK = 32, kStages = 3, kOperands = 4, kGroup = 4;
};

template <int KIND>
constexpr size_t smem_bytes() {
  return static_cast<size_t>(Cfg<KIND>::kStages) * Cfg<KIND>::kOperands * kOperandBytes;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ float to_tf32(float v) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(v));
  return __uint_as_float(r);
}

// Stage one operand's chunk: rows [row0, row0 + 128) x K [k0, k0 + kK) of X, 8 groups per thread.
template <int KIND>
__device__ __forceinline__ void stage_operand(const float* X, long long rs, long long ks, int row0, int rows, int k0,
                                              int K, unsigned char* hi, unsigned char* lo, int p) {
  using C = Cfg<KIND>;
  constexpr int kGroupsPerRow = C::kK / C::kGroup;  // 8
  constexpr int kPer = kTile * kGroupsPerRow / 128;  // groups per producer thread: 8
  const bool k_contig = ks == 1;
  // The loads of a batch of groups are all issued before the first shared-memory store: the stores
  // go through generic pointers the compiler cannot tell apart from X, so a load placed after a
  // store would wait for it, and the chunk would cost one global round trip per group.
  constexpr int kBatch = KIND == 1 ? 4 : 8;  // groups in flight: 32 floats either way
#pragma unroll
  for (int b0 = 0; b0 < kPer; b0 += kBatch) {
    float v[kBatch][C::kGroup];
#pragma unroll
    for (int ib = 0; ib < kBatch; ++ib) {
      const int g = (b0 + ib) * 128 + p;
      const int row = k_contig ? g / kGroupsPerRow : g % kTile;
      const int kg = k_contig ? g % kGroupsPerRow : g / kTile;
      const int gr = row0 + row;
#pragma unroll
      for (int e = 0; e < C::kGroup; ++e) {
        const int gk = k0 + kg * C::kGroup + e;
        v[ib][e] = (gr < rows && gk < K) ? X[gr * rs + gk * ks] : 0.0f;
      }
    }
#pragma unroll
    for (int ib = 0; ib < kBatch; ++ib) {
      const int g = (b0 + ib) * 128 + p;
      const int row = k_contig ? g / kGroupsPerRow : g % kTile;
      const int kg = k_contig ? g % kGroupsPerRow : g / kTile;
      const uint32_t off = tc::kmajor_offset(row, kg * C::kGroup, C::kK, KIND == 1 ? 2 : 4);
      if constexpr (KIND == 1) {
        uint4 w;
        __nv_bfloat162 q0 = __floats2bfloat162_rn(v[ib][0], v[ib][1]), q1 = __floats2bfloat162_rn(v[ib][2], v[ib][3]);
        __nv_bfloat162 q2 = __floats2bfloat162_rn(v[ib][4], v[ib][5]), q3 = __floats2bfloat162_rn(v[ib][6], v[ib][7]);
        w.x = *reinterpret_cast<uint32_t*>(&q0);
        w.y = *reinterpret_cast<uint32_t*>(&q1);
        w.z = *reinterpret_cast<uint32_t*>(&q2);
        w.w = *reinterpret_cast<uint32_t*>(&q3);
        *reinterpret_cast<uint4*>(hi + off) = w;
      } else {
        float h[4], l[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          h[e] = to_tf32(v[ib][e]);
          l[e] = to_tf32(v[ib][e] - h[e]);
        }
        *reinterpret_cast<float4*>(hi + off) = make_float4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<float4*>(lo + off) = make_float4(l[0], l[1], l[2], l[3]);
      }
    }
  }
}

template <int KIND>
__global__ void __launch_bounds__(kThreads, 1) k_gemm_ws(WsGemmArgs g) {
  using C = Cfg<KIND>;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t full[C::kStages], empty[C::kStages], done;
  __shared__ uint32_t tmem_base;
  __shared__ int s_fail;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int tr = blockIdx.y, tn = blockIdx.x;
  if (g.lower) {  // CTA t -> the t-th lower tile in row order: (I, J), J <= I
    int I = 0;
    while ((I + 1) * (I + 2) / 2 <= static_cast<int>(blockIdx.x)) ++I;
    tr = I;
    tn = blockIdx.x - I * (I + 1) / 2;
  }
  const int r0 = tr * kTile, n0 = tn * kTile;
  const int nk = (g.K + C::kK - 1) / C::kK;
  if (warp == 0) tc::tmem_alloc(&tmem_base, kTile);
  if (tid == 0) {
    for (int s = 0; s < C::kStages; ++s) {
      tc::mbar_init(&full[s], 128);
      tc::mbar_init(&empty[s], 1);
    }
    tc::mbar_init(&done, 1);
    s_fail = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tmem = tmem_base;
  auto stage_ptr = [&](int s, int operand) { return smem + (static_cast<size_t>(s) * C::kOperands + operand) * kOperandBytes; };
  bool ok = true;
  if (warp < 4) {
    // ---- producers ----
    for (int kc = 0; kc < nk && ok; ++kc) {
      const int s = kc % C::kStages;
      if (kc >= C::kStages && !tc::mbar_wait(&empty[s], ((kc / C::kStages) - 1) & 1, kWaitLimit)) {
        ok = false;
        break;
      }
      const int k0 = kc * C::kK;
      if constexpr (KIND == 1) {
        stage_operand<1>(g.A, g.a_rs, g.a_ks, r0, g.M, k0, g.K, stage_ptr(s, 0), nullptr, tid);
        stage_operand<1>(g.B, g.b_rs, g.b_ks, n0, g.N, k0, g.K, stage_ptr(s, 1), nullptr, tid);
      } else {
        stage_operand<0>(g.A, g.a_rs, g.a_ks, r0, g.M, k0, g.K, stage_ptr(s, 0), stage_ptr(s, 1), tid);
        stage_operand<0>(g.B, g.b_rs, g.b_ks, n0, g.N, k0, g.K, stage_ptr(s, 2), stage_ptr(s, 3), tid);
      }
      tc::fence_async_smem();  // generic-proxy stores -> visible to the tensor cores
      mbar_arrive(&full[s]);
    }
    if (!ok) atomicExch(&s_fail, 1);
    __syncwarp();
  } else if (lane == 0) {
    // ---- MMA issue ----
    constexpr uint32_t idesc = tc::instr_desc(KIND == 1 ? 1 : 2, kTile, kTile);
    constexpr uint32_t lbo = 128, sbo = 1024;
    for (int kc = 0; kc < nk; ++kc) {
      const int s = kc % C::kStages;
      if (!tc::mbar_wait(&full[s], (kc / C::kStages) & 1, kWaitLimit)) {
        ok = false;
        break;
      }
      tc::fence_after();
      if constexpr (KIND == 1) {
        const uint32_t a = tc::smem_u32(stage_ptr(s, 0)), b = tc::smem_u32(stage_ptr(s, 1));
#pragma unroll
        for (int q = 0; q < C::kK / 16; ++q) {
          const uint32_t o = static_cast<uint32_t>(q) * 256;
          tc::mma<1>(tmem, tc::smem_desc(a + o, lbo, sbo), tc::smem_desc(b + o, lbo, sbo), idesc, (kc > 0 || q > 0));
        }
      } else {
        const uint32_t ah = tc::smem_u32(stage_ptr(s, 0)), al = tc::smem_u32(stage_ptr(s, 1));
        const uint32_t bh = tc::smem_u32(stage_ptr(s, 2)), bl = tc::smem_u32(stage_ptr(s, 3));
#pragma unroll
        for (int q = 0; q < C::kK / 8; ++q) {
          const uint32_t o = static_cast<uint32_t>(q) * 256;
          tc::mma<0>(tmem, tc::smem_desc(ah + o, lbo, sbo), tc::smem_desc(bh + o, lbo, sbo), idesc, (kc > 0 || q > 0));
          tc::mma<0>(tmem, tc::smem_desc(ah + o, lbo, sbo), tc::smem_desc(bl + o, lbo, sbo), idesc, 1);
          tc::mma<0>(tmem, tc::smem_desc(al + o, lbo, sbo), tc::smem_desc(bh + o, lbo, sbo), idesc, 1);
        }
      }
      tc::commit(&empty[s]);
    }
    tc::commit(&done);  // arrives once every MMA issued above has completed (or at once if none)
    if (!ok) atomicExch(&s_fail, 1);
  }
  __syncwarp();
  // ---- epilogue (warps 0-3) ----
  bool have = false;
  if (warp < 4) {
    have = tc::mbar_wait(&done, 0, kWaitLimit);
    tc::fence_after();
  }
  __syncwarp();
  __syncthreads();
  const bool fine = have && s_fail == 0;
  if (warp < 4) {
    if (fine) {
      const int r = r0 + warp * 32 + lane;
#pragma unroll 1
      for (int cc = 0; cc < kTile / 32; ++cc) {
        float v[32];
        tc::tmem_ld32(tmem + (static_cast<uint32_t>(warp * 32) << 16) + cc * 32, v);
        if (r < g.M) {
          // the 32 old values of C are read before the first store (a read after a store to
          // a possibly aliasing address would wait for it: one round trip per column)
          float old[32];
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const int n = n0 + cc * 32 + c;
            old[c] = (g.beta != 0.0f && n < g.N) ? g.C[r * g.c_rs + n * g.c_cs] : 0.0f;
          }
#pragma unroll
          for (int c = 0; c < 32; ++c) {
            const int n = n0 + cc * 32 + c;
            if (n >= g.N) continue;
            float out = g.alpha * (nk > 0 ? v[c] : 0.0f);
            if (g.beta != 0.0f) out += g.beta * old[c];
            if (g.bias) out += g.bias[n];
            if (g.relu) out = fmaxf(out, 0.0f);
            g.C[r * g.c_rs + n * g.c_cs] = out;
          }
        }
      }
    } else if (tid == 0) {
      atomicExch(g.err, 3);
      tc::mbar_wait(&done, 0, kWaitLimit);  // MMAs in flight finish before TMEM is released
    }
  }
  __syncwarp();
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, kTile);
}

}  // namespace wsg

// Launch: one CTA per output tile (per lower tile when g.lower).
template <int KIND>
inline void launch_gemm_ws(const WsGemmArgs& g, cudaStream_t st) {
  const size_t smem = wsg::smem_bytes<KIND>();
  once_per_device((const void*)wsg::k_gemm_ws<KIND>, [&] {
    SOV_CUDA(cudaFuncSetAttribute(wsg::k_gemm_ws<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  });
  const int tm = ceil_div(g.M, wsg::kTile), tn = ceil_div(g.N, wsg::kTile);
  dim3 grid = g.lower ? dim3(tm * (tm + 1) / 2) : dim3(tn, tm);
  wsg::k_gemm_ws<KIND><<<grid, wsg::kThreads, smem, st>>>(g);
  SOV_LAUNCH_CHECK();
}

}  // namespace sov
