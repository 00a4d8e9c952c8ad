// band.cuh -- banded LDL^T of the normal matrix (natural order), for small half-bandwidths.
#pragma once

#include <cuda_runtime.h>

namespace sov {

constexpr int kBandMax = 8;  // largest half-bandwidth the band kernels take

struct BandSystem {
  double* B;     // (kd + 1) x m, B[off * m + col] = M[col + off][col]
  double* dinv;  // m: 1 / D
  double* diag;  // m: assembled diagonal (pivot-drop reference)
  int m, kd;
  int* drop_count;
  int* fail;
};

// B must be padded so that the template width (>= kd) never reads past the allocation:
// allocate (kBandMax + 1) * m doubles and zero the unused diagonals once.
void band_factor(const BandSystem& s, cudaStream_t st, int* launches);
void band_solve(const BandSystem& s, double* z, cudaStream_t st, int* launches);

}  // namespace sov
