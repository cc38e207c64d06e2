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

// One step of the device-side SP2 stopping rule (Sp2State, Sp2Rule in kernels.hpp), run by
// a single thread after the step's traces are in state: records the step's error, and on
// convergence, the rounding floor, a non-finite error or the step cap sets
// state[kSp2Stop] = step (later steps then do nothing) and state[kSp2Ok].
template <class Rule>
__device__ __forceinline__ void sp2_control(double *state, int step, double e, const Rule &rule) {
  constexpr int kStop = 4, kOk = 5, kRing = 6;
  const double prev2 = step >= 2 ? state[kRing + (step + 1) % 3] : 0.0;  // error two steps before
  state[kRing + step % 3] = e;
  int stop = 0, ok = 0;
  if (!isfinite(e)) {
    stop = 1;
  } else if (fabs(e) <= rule.tol_done) {
    stop = ok = 1;
  } else if (step >= 2 && fabs(e) < rule.tol_floor && fabs(e) >= fabs(prev2)) {
    stop = ok = 1;  // no further progress at the rounding floor
  } else if (step + 1 >= rule.max_steps) {
    stop = 1;
  }
  if (stop) {
    state[kStop] = (double)step;
    state[kOk] = (double)ok;
  }
}

// Whether step `step` of a purification still runs (no earlier step stopped it).
__device__ __forceinline__ bool sp2_active(const double *state, int step) {
  return state == nullptr || (double)step <= state[4];
}

}  // namespace pm7
