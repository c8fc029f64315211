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

// a / b as the point-wise step evaluates it: the hardware's approximate
// reciprocal (rcp.approx, relative error below 2^-23) refined by one
// Newton-Raphson step with FMA, then the quotient corrected by its FMA
// residual (Markstein's division; Muller et al., Handbook of Floating-Point
// Arithmetic, 2nd ed., section 4.6). For normal operands with a normal
// quotient the result is within one ulp of a / b and nearly always the
// correctly rounded quotient; here b = |y| + 1e-12 >= 1e-12 and a is an
// amplitude or a magnitude, so the quotient is never subnormal and a = 0
// gives 0. Unlike the IEEE division it has no slow path, which in the
// unrolled passes costs registers and spills.
__device__ __forceinline__ float divide(float a, float b) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(b));
  const float e = fmaf(-b, y, 1.0f);
  y = fmaf(e, y, y);
  const float q = a * y;
  const float r = fmaf(-b, q, a);
  return fmaf(r, y, q);
}

// sqrt(x) for finite x >= 0 as the point-wise step evaluates it: the
// hardware's approximate reciprocal square root y (rsqrt.approx, relative
// error below 2^-22), s = x y, then one Newton-Raphson correction of s by its
// FMA residual x - s^2 (Markstein's square root; Muller et al., Handbook of
// Floating-Point Arithmetic, 2nd ed., section 5.4). The result is within one
// ulp of the IEEE square root and nearly always equal to it. Inputs below
// 2^-64 are scaled by 2^64 first (and the root by 2^-32 after), so that
// subnormal operands are neither flushed nor lost; x = 0 gives 0. Like
// divide(), it has no slow path.
__device__ __forceinline__ float square_root(float x) {
  const bool tiny = x < 0x1p-64f;
  const float xs = tiny ? x * 0x1p64f : x;
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(xs));
  const float s = xs * y;
  const float r = fmaf(-s, s, xs);
  const float q = fmaf(r, 0.5f * y, s);
  return xs > 0.0f ? (tiny ? q * 0x1p-32f : q) : 0.0f;
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
  // The reference's expression (src/cuda/device.cuh:20-27): the square root
  // of the squared magnitude and the quotient by (|y| + eps), each within one
  // ulp of the IEEE operation.
  const float mag = square_root(re * re + im * im);
  float f;
  if constexpr (M == Mode::kGrad) {
    f = 0.0f;
    if (a >= 0.0f) {
      const float d = mag - a;
      acc += d * d;
      f = 2.0f * (1.0f - divide(a, mag + kEps)) * out_scale;
    }
  } else {
    float target = mag;
    if (a >= 0.0f) {
      const float d = mag - a;
      acc += d * d;
      target = a;
    }
    f = divide(target, mag + kEps) * out_scale;
  }
  return {re * f, im * f};
}

template <Mode M>
__device__ __forceinline__ float2 pointwise_projection(float2 v, float a, float s, float& acc) {
  return pointwise_projection<M>(v, a, s, acc, s);
}

}  // namespace qpb
