// sx_kernels.cuh -- device helpers shared by the kernel files.
#pragma once

#include "sx_internal.h"

namespace sx {

// Per-system descriptor for batched factorisation / band sweeps.
struct SysDesc {
  double *tiles;  // nblk*(J+1)*TSZ
  double *dinv;   // nblk*TSZ
  int nblk, J;
  int *status;
  const int *jb;  // tiles right of the diagonal in each block row (null: J)
};

// Address of U(m, n), m <= n, n - m <= kd, inside the tile array.
__host__ __device__ __forceinline__ size_t tile_addr(int m, int n, int J) {
  const int bm = m / NB, bn = n / NB;
  return ((size_t)bn * (J + 1) + (bn - bm)) * TSZ + (size_t)(m - bm * NB) * LDT + (n - bn * NB);
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sumf(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Factor the systems' bands, all systems in each launch; sync = false
// returns without waiting (statuses to be checked after st completes).
int factor_batch(std::vector<System *> &systems, cudaStream_t st, bool sync = true);

}  // namespace sx
