// Device point-wise step shared by the modulus and loss-gradient line passes.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "common.cuh"
#include "line_pass.cuh"

namespace qpb {

// An amplitude in its storage type (float, __half or __nv_bfloat16) as float.
template <class AmpT>
__device__ __forceinline__ float to_float(AmpT a) {
  if constexpr (std::is_same_v<AmpT, float>) {
    return a;
  } else if constexpr (std::is_same_v<AmpT, __half>) {
    return __half2float(a);
  } else {
    return __bfloat162float(a);
  }
}

// The point-wise step of a modulus (kMod) or amplitude-loss gradient (kGrad)
// pass on one element of the unnormalised forward transform. `s` = 1/sqrt(n)
// scales it to the unitary transform and prepares the unnormalised inverse; `a`
// is the amplitude, negative on masked pixels. Adds (|y| - A)^2 to `acc` on
// usable pixels. kMod follows src/cuda/device.cuh:17-29 of the reference
// (target A, masked pixels scaled by |y| / (|y| + eps)); kGrad returns
// 2 (y - P_M y) = 2 (1 - A / (|y| + eps)) y on usable pixels and 0 on masked
// ones, whose inverse transform is the gradient of sum (|F x| - A)^2 in
// PyTorch's convention (dL/dRe + i dL/dIm).
//   `out_scale` multiplies the result (s unless the caller defers the inverse's
// 1/sqrt(n) to after the inverse transform, as the fp16 wave storage does to
// keep stored values in range: src/cuda/device.cuh:14-16 of the reference).
template <Mode M>
__device__ __forceinline__ float2 pointwise_projection(float2 v, float a, float s, float& acc,
                                                       float out_scale) {
  const float re = v.x * s;
  const float im = v.y * s;
  // The reference's own expression, rounded the same way: an IEEE square root
  // of the squared magnitude and an IEEE division by (|y| + eps).
  const float mag = sqrtf(re * re + im * im);
  float f;
  if constexpr (M == Mode::kGrad) {
    f = 0.0f;
    if (a >= 0.0f) {
      const float d = mag - a;
      acc += d * d;
      f = 2.0f * (1.0f - a / (mag + kEps)) * out_scale;
    }
  } else {
    float target = mag;
    if (a >= 0.0f) {
      const float d = mag - a;
      acc += d * d;
      target = a;
    }
    f = target / (mag + kEps) * out_scale;
  }
  return {re * f, im * f};
}

template <Mode M>
__device__ __forceinline__ float2 pointwise_projection(float2 v, float a, float s, float& acc) {
  return pointwise_projection<M>(v, a, s, acc, s);
}

}  // namespace qpb
