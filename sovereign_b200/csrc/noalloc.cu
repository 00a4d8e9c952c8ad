// noalloc.cu -- sov_normal_factor_solve_noalloc: the dense FP64 normal-equation factor and solve
// for callers that cannot let a library allocate device memory.
//
// Some host applications own every byte of device memory themselves (their own pool, or a
// process running close to the memory limit) and hand a library only buffers they already
// allocated. For them this entry point takes device pointers for all inputs and outputs and uses,
// for its working storage, one file-scope device array of fixed size: the normal matrix (up to
// kNoAllocMaxRows rows, padded to a multiple of 64), the inverted diagonal blocks, the padded
// solve vector, the assembled diagonal, the dataflow flags and the counters. It never calls
// cudaMalloc, cudaFree or any allocating routine.
//
// The array lives in every GPU that loads the library until the process exits. Its address is
// looked up with cudaGetSymbolAddress on the first call on each device (with that device
// current); that first call should therefore come before any stream capture on that device.
// Every call reuses the same array and leaves its contents behind, so each call clears what must
// start at zero, and two calls whose work overlaps on the GPU (different streams, or different
// host threads) race on the array: callers must order them.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>

#include "common.cuh"
#include "dense.cuh"
#include "sov_ipm.h"

namespace sov {
namespace {

constexpr int kNoAllocMaxRows = SOV_NOALLOC_MAX_ROWS;  // 512
constexpr int kNoAllocMaxBlocks = kNoAllocMaxRows / kNB;
constexpr size_t kScratchM = static_cast<size_t>(kNoAllocMaxRows) * kNoAllocMaxRows;
constexpr size_t kScratchLinv = static_cast<size_t>(kNoAllocMaxBlocks) * kNB * kNB;
constexpr size_t kScratchDoubles = kScratchM + kScratchLinv + 2 * kNoAllocMaxRows;
constexpr int kScratchInts = 64 + 8;  // flags (up to 64 blocks) + counters

static __device__ __align__(256) double g_scratch[kScratchDoubles];
static __device__ __align__(256) int g_scratch_int[kScratchInts];

struct ScratchPtrs {
  double* d = nullptr;
  int* i = nullptr;
};

std::mutex g_mu;
std::map<int, ScratchPtrs> g_ptrs;  // per device

int resolve(int dev, ScratchPtrs& out) {
  std::lock_guard<std::mutex> g(g_mu);
  auto it = g_ptrs.find(dev);
  if (it != g_ptrs.end()) {
    out = it->second;
    return SOV_OK;
  }
  ScratchPtrs p;
  if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p.d), g_scratch) != cudaSuccess) return SOV_E_CUDA;
  if (cudaGetSymbolAddress(reinterpret_cast<void**>(&p.i), g_scratch_int) != cudaSuccess) return SOV_E_CUDA;
  g_ptrs[dev] = p;
  out = p;
  return SOV_OK;
}

// M (column-major, leading dimension ld, lower triangle) += a_p d_k a_q for every pair of
// entries p, q of column k; rows within a column must be distinct. The caller's device arrays
// were never seen by the host, so a column whose col_ptr decreases and an entry whose row lies
// outside [0, m) are skipped and counted in *bad instead of being written.
__global__ void k_scatter_normal(int n, int m, const int* __restrict__ cp, const int* __restrict__ ri,
                                 const double* __restrict__ v, const double* __restrict__ d, double* M, int ld,
                                 int* bad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int p0 = cp[k], p1 = cp[k + 1];
  if (p0 < 0 || p1 < p0) {
    atomicAdd(bad, 1);
    return;
  }
  const double dk = d[k];
  for (int p = p0; p < p1; ++p) {
    const int rp = ri[p];
    if (rp < 0 || rp >= m) {
      atomicAdd(bad, 1);
      continue;
    }
    for (int q = p0; q <= p; ++q) {
      const int rq = ri[q];
      if (rq < 0 || rq >= m) continue;  // counted once, as entry p
      const int r = max(rp, rq), c = min(rp, rq);
      atomicAdd(M + static_cast<int64_t>(c) * ld + r, v[p] * dk * v[q]);
    }
  }
}

// diag[i] = M_ii + 1e-12 (interior_point.cpp:96-100); padding rows get the identity.
__global__ void k_finish_diag(double* M, int m, int mp, double* diag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= mp) return;
  double* mii = M + static_cast<int64_t>(i) * mp + i;
  if (i < m) {
    *mii += 1e-12;
    diag[i] = *mii;
  } else {
    *mii = 1.0;
  }
}

__global__ void k_copy_pad(const double* src, double* dst, int m, int mp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < mp) dst[i] = i < m ? src[i] : 0.0;
}

__global__ void k_copy_back(const double* src, double* dst, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) dst[i] = src[i];
}

}  // namespace
}  // namespace sov

extern "C" int sov_normal_factor_solve_noalloc(int32_t m, int32_t n, const int32_t* col_ptr, const int32_t* row_idx,
                                               const double* values, const double* d, double* rhs, int32_t nrhs,
                                               int32_t* dropped_pivots, void* cuda_stream) {
  using namespace sov;
  if (m <= 0 || n < 0 || nrhs < 0 || !col_ptr || !d || !rhs || (n > 0 && (!row_idx || !values)))
    return record_error(SOV_E_ARGUMENT, "noalloc factor/solve: null array or negative size");
  if (m > kNoAllocMaxRows)
    return record_error(SOV_E_TOO_LARGE, "noalloc factor/solve: m = " + std::to_string(m) + " exceeds the fixed "
                                             "working array (m <= " + std::to_string(kNoAllocMaxRows) + ")");
  if (int rc = require_device()) return rc;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return record_error(SOV_E_NO_DEVICE, "noalloc factor/solve: no device");
  ScratchPtrs sp;
  if (resolve(dev, sp) != SOV_OK)
    return record_error(SOV_E_CUDA, "noalloc factor/solve: cudaGetSymbolAddress of the working array failed");
  cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
  try {
    const int nb = ceil_div(m, kNB), mp = nb * kNB;
    double* M = sp.d;
    double* Linv = sp.d + kScratchM;
    double* z = Linv + kScratchLinv;
    double* diag = z + kNoAllocMaxRows;
    unsigned* flags = reinterpret_cast<unsigned*>(sp.i);
    // [0] dropped pivots, [1] non-finite pivot, [2] solve timeout, [3] tickets, [4] bad entries
    int* counters = sp.i + 64;
    // clear what must start at zero: the matrix, the flags and the counters
    SOV_CUDA(cudaMemsetAsync(M, 0, sizeof(double) * static_cast<size_t>(mp) * mp, st));
    SOV_CUDA(cudaMemsetAsync(sp.i, 0, sizeof(int) * kScratchInts, st));
    if (n > 0) k_scatter_normal<<<ceil_div(n, 128), 128, 0, st>>>(n, m, col_ptr, row_idx, values, d, M, mp, counters + 4);
    SOV_LAUNCH_CHECK();
    int bad = 0;
    SOV_CUDA(cudaMemcpyAsync(&bad, counters + 4, sizeof(int), cudaMemcpyDeviceToHost, st));
    SOV_CUDA(cudaStreamSynchronize(st));
    if (bad)
      return record_error(SOV_E_ARGUMENT, "noalloc factor/solve: " + std::to_string(bad) +
                                              " column(s) or entries with col_ptr decreasing or a row outside [0, m)");
    k_finish_diag<<<ceil_div(mp, 128), 128, 0, st>>>(M, m, mp, diag);
    SOV_LAUNCH_CHECK();
    DenseSystem<double> s{M, Linv, diag, m, mp, nb, counters, counters + 1, flags,
                          reinterpret_cast<unsigned*>(counters + 3), 1e-13};
    dense_cholesky<double>(s, st, nullptr);
    unsigned epoch = 0;
    for (int r = 0; r < nrhs; ++r) {
      double* col = rhs + static_cast<size_t>(r) * m;
      k_copy_pad<<<ceil_div(mp, 128), 128, 0, st>>>(col, z, m, mp);
      dense_solve<double>(s, z, epoch, counters + 2, st, nullptr);
      k_copy_back<<<ceil_div(m, 128), 128, 0, st>>>(z, col, m);
    }
    int h[3] = {0, 0, 0};
    SOV_CUDA(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    SOV_CUDA(cudaStreamSynchronize(st));
    if (dropped_pivots) *dropped_pivots = h[0];
    if (h[1]) return record_error(SOV_E_NUMERICAL, "noalloc factor/solve: non-finite pivot");
    if (h[2]) return record_error(SOV_E_CUDA, "noalloc factor/solve: a triangular-solve wait ran out");
  } catch (const std::exception& e) {
    return record_error(SOV_E_CUDA, std::string("noalloc factor/solve: ") + e.what());
  }
  return SOV_OK;
}
