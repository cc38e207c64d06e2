// Shared device helpers: deterministic block reductions and error checks.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>

namespace pm7 {

// Sum of `v` over the whole block (1-, 2- or 3-D, BLOCK threads), returned on the
// block's first thread. The combine order is fixed by thread index, so the result
// is the same on every run (no atomics).
template <int BLOCK>
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double warp_part[BLOCK / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int lane = tid & 31, wid = tid >> 5;
  if (lane == 0) warp_part[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (tid == 0) {
    for (int w = 0; w < BLOCK / 32; ++w) s += warp_part[w];
  }
  __syncthreads();
  return s;
}

}  // namespace pm7
