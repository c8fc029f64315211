// Device point-wise step shared by the modulus and loss-gradient line passes.
#pragma once

#include "common.cuh"
#include "line_pass.cuh"

namespace qpb {

// The point-wise step of a modulus (kMod) or amplitude-loss gradient (kGrad)
// pass on one element of the unnormalised forward transform. `s` = 1/sqrt(n)
// scales it to the unitary transform and prepares the unnormalised inverse; `a`
// is the amplitude, negative on masked pixels. Adds (|y| - A)^2 to `acc` on
// usable pixels. kMod follows src/cuda/device.cuh:17-29 of the reference
// (target A, masked pixels scaled by |y| / (|y| + eps)); kGrad returns
// 2 (y - P_M y) = 2 (1 - A / (|y| + eps)) y on usable pixels and 0 on masked
// ones, whose inverse transform is the gradient of sum (|F x| - A)^2 in
// PyTorch's convention (dL/dRe + i dL/dIm).
template <Mode M>
__device__ __forceinline__ float2 pointwise_projection(float2 v, float a, float s, float& acc) {
  const float re = v.x * s;
  const float im = v.y * s;
  const float mag = sqrtf(re * re + im * im);
  float f;
  if constexpr (M == Mode::kGrad) {
    f = 0.0f;
    if (a >= 0.0f) {
      const float d = mag - a;
      acc += d * d;
      f = 2.0f * (1.0f - __fdividef(a, mag + kEps)) * s;
    }
  } else {
    float target = mag;
    if (a >= 0.0f) {
      const float d = mag - a;
      acc += d * d;
      target = a;
    }
    // approximate division (<= 2 ulp): branch-free, far inside the tolerances
    f = __fdividef(target, mag + kEps) * s;
  }
  return {re * f, im * f};
}

}  // namespace qpb
