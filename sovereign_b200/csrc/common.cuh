// common.cuh -- shared device helpers and error handling for the B200 interior-point engine.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

#include "errors.hpp"

namespace sov {

struct CudaError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

#define SOV_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t sov_err_ = (call);                                                       \
    if (sov_err_ != cudaSuccess)                                                         \
      throw ::sov::CudaError(std::string(#call) + ": " + cudaGetErrorString(sov_err_));  \
  } while (0)

#define SOV_LAUNCH_CHECK() SOV_CUDA(cudaGetLastError())

constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(kFull, v, o));
  return v;
}

// Block-wide reduction of NV values at once (sum / max / min chosen per slot by `ops`,
// 0 = sum, 1 = max, 2 = min). `scratch` needs NV * 32 doubles. Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], const int (&ops)[NV], double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = ops[k] == 0 ? warp_sum(v[k]) : ops[k] == 1 ? warp_max(v[k]) : warp_min(v[k]);
  __syncthreads();
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) scratch[k * 32 + warp] = v[k];
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      const double id = ops[k] == 0 ? 0.0 : ops[k] == 1 ? -INFINITY : INFINITY;
      double t = lane < nwarps ? scratch[k * 32 + lane] : id;
      v[k] = ops[k] == 0 ? warp_sum(t) : ops[k] == 1 ? warp_max(t) : warp_min(t);
    }
  }
  __syncthreads();
}

// Acquire / release flag accesses for the dataflow triangular solves.
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Runs fn() once per (current device, key), thread-safe: kernel attributes such as the opt-in to
// more than 48 KB of dynamic shared memory are set per device, so every device gets its own call,
// and host threads that launch concurrently wait for the first one's call to finish.
inline std::mutex& once_mutex() {
  static std::mutex m;
  return m;
}
inline std::set<std::pair<int, const void*>>& once_done() {
  static std::set<std::pair<int, const void*>> s;
  return s;
}
template <class F>
void once_per_device(const void* key, F&& fn) {
  int dev = 0;
  SOV_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(once_mutex());
  if (once_done().count({dev, key})) return;
  fn();
  once_done().insert({dev, key});
}
constexpr int kMaxDevices = 64;

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

}  // namespace sov
