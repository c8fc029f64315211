// Storage types of the wave and the iterate: complex64 (float2) or two fp16
// halves (__half2, the reference's fp16 path, src/cuda/half.cu:14-83). The
// line passes compute in FP32 either way; a half2 element is widened on load
// and rounded to nearest on store.
#pragma once

#include <cuda_fp16.h>

#include <type_traits>

namespace qpb {

template <class T>
__device__ __forceinline__ float2 load_c(const T& v) {
  if constexpr (std::is_same_v<T, float2>) {
    return v;
  } else {
    return __half22float2(v);
  }
}

template <class T>
__device__ __forceinline__ T store_c(float2 v) {
  if constexpr (std::is_same_v<T, float2>) {
    return v;
  } else {
    return __float22half2_rn(v);
  }
}

template <class T>
inline constexpr bool kHalfStorage = std::is_same_v<T, __half2>;

}  // namespace qpb
