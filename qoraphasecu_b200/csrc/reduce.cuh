// Warp and block reductions used by the fused passes.
#pragma once

#include <cuda_runtime.h>

namespace qpb {

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_sum_double(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum over the block, valid in thread 0. Every thread of the block must call
// it; blockDim.x is a multiple of 32 and at most 1024. AGAIN keeps the closing
// barrier that a second call in the same block needs; either way the call
// holds one block barrier after every thread has entered it.
template <bool AGAIN = true>
__device__ __forceinline__ double block_sum_double(double v) {
  __shared__ double partial[32];
  v = warp_sum_double(v);
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (lane == 0) partial[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < static_cast<int>(blockDim.x >> 5) ? partial[lane] : 0.0;
    v = warp_sum_double(v);
  }
  if constexpr (AGAIN) __syncthreads();
  return v;
}

}  // namespace qpb
