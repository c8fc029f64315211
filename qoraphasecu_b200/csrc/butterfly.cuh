// In-register DFT butterflies of radix 2, 3, 4, 5, 8 and 16.
//
// Forward uses W = exp(-2 pi i / R); INV flips the sign of every imaginary
// unit. Outputs are in natural order: v[m] <- sum_q v[q] W^{q m}. Constants
// are the exact values of cos/sin at the DFT angles.
#pragma once

#include "common.cuh"

namespace qpb {

// a * (-i) forward, a * (+i) inverse: the product with W_4^1.
template <bool INV>
__device__ __forceinline__ float2 mul_w4(float2 a) {
  return INV ? mul_pi(a) : mul_mi(a);
}

template <bool INV>
__device__ __forceinline__ void bfly2(float2& a, float2& b) {
  const float2 t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <bool INV>
__device__ __forceinline__ void bfly4(float2& v0, float2& v1, float2& v2, float2& v3) {
  const float2 t0 = cadd(v0, v2);
  const float2 t1 = csub(v0, v2);
  const float2 t2 = cadd(v1, v3);
  const float2 t3 = mul_w4<INV>(csub(v1, v3));
  v0 = cadd(t0, t2);
  v2 = csub(t0, t2);
  v1 = cadd(t1, t3);
  v3 = csub(t1, t3);
}

template <bool INV>
__device__ __forceinline__ void bfly3(float2& v0, float2& v1, float2& v2) {
  constexpr float kS = 0.86602540378443864676f;  // sin(2 pi / 3)
  const float2 t = cadd(v1, v2);
  const float2 m = cadd(v0, cscale(t, -0.5f));
  // (v1 - v2) * (-i sin) forward, (+i sin) inverse
  const float2 d = cscale(csub(v1, v2), kS);
  const float2 s = mul_w4<INV>(d);
  v0 = cadd(v0, t);
  v1 = cadd(m, s);
  v2 = csub(m, s);
}

template <bool INV>
__device__ __forceinline__ void bfly5(float2& v0, float2& v1, float2& v2, float2& v3, float2& v4) {
  constexpr float c1 = 0.30901699437494742410f;   // cos(2 pi / 5)
  constexpr float c2 = -0.80901699437494742410f;  // cos(4 pi / 5)
  constexpr float s1 = 0.95105651629515357212f;   // sin(2 pi / 5)
  constexpr float s2 = 0.58778525229247312917f;   // sin(4 pi / 5)
  const float2 a1 = cadd(v1, v4);
  const float2 a2 = cadd(v2, v3);
  const float2 b1 = csub(v1, v4);
  const float2 b2 = csub(v2, v3);
  const float2 r1 = {v0.x + c1 * a1.x + c2 * a2.x, v0.y + c1 * a1.y + c2 * a2.y};
  const float2 r2 = {v0.x + c2 * a1.x + c1 * a2.x, v0.y + c2 * a1.y + c1 * a2.y};
  // i-parts: forward X1 = r1 - i (s1 b1 + s2 b2), X2 = r2 - i (s2 b1 - s1 b2)
  const float2 q1 = mul_w4<INV>({s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y});
  const float2 q2 = mul_w4<INV>({s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y});
  v0 = cadd(v0, cadd(a1, a2));
  v1 = cadd(r1, q1);
  v4 = csub(r1, q1);
  v2 = cadd(r2, q2);
  v3 = csub(r2, q2);
}

// Multiply by W_8^1 = (1 - i)/sqrt(2) forward, (1 + i)/sqrt(2) inverse.
template <bool INV>
__device__ __forceinline__ float2 mul_w8(float2 a) {
  constexpr float r = 0.70710678118654752440f;
  return INV ? float2{(a.x - a.y) * r, (a.x + a.y) * r} : float2{(a.x + a.y) * r, (a.y - a.x) * r};
}

// Multiply by W_8^3 = (-1 - i)/sqrt(2) forward, (-1 + i)/sqrt(2) inverse.
template <bool INV>
__device__ __forceinline__ float2 mul_w8_3(float2 a) {
  constexpr float r = 0.70710678118654752440f;
  return INV ? float2{(-a.x - a.y) * r, (a.x - a.y) * r} : float2{(a.y - a.x) * r, (-a.x - a.y) * r};
}

// v[0..7] in natural order.
template <bool INV>
__device__ __forceinline__ void bfly8(float2* v) {
  // even / odd 4-point DFTs
  float2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  float2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  bfly4<INV>(e0, e1, e2, e3);
  bfly4<INV>(o0, o1, o2, o3);
  o1 = mul_w8<INV>(o1);
  o2 = mul_w4<INV>(o2);
  o3 = mul_w8_3<INV>(o3);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// v[0..15] in natural order: 4 x 4 with W_16 twiddles between the two levels.
template <bool INV>
__device__ __forceinline__ void bfly16(float2* v) {
  constexpr float c1 = 0.92387953251128675613f;  // cos(pi / 8)
  constexpr float s1 = 0.38268343236508977173f;  // sin(pi / 8)
  constexpr float r = 0.70710678118654752440f;
  // Level 1: for each n1 in 0..3, a 4-point DFT over v[n1 + 4 n2].
  for (int n1 = 0; n1 < 4; ++n1) bfly4<INV>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
  // Twiddles W_16^{n1 k2} on v[n1 + 4 k2].
  const float sg = INV ? 1.0f : -1.0f;
  const float2 w1 = {c1, sg * s1};   // W^1
  const float2 w2 = {r, sg * r};     // W^2
  const float2 w3 = {s1, sg * c1};   // W^3
  const float2 w6 = {-r, sg * r};    // W^6
  const float2 w9 = {-c1, -sg * s1};  // W^9 = -W^1
  v[5] = cmul(v[5], w1);
  v[9] = cmul(v[9], w2);
  v[13] = cmul(v[13], w3);
  v[6] = cmul(v[6], w2);
  v[10] = mul_w4<INV>(v[10]);  // W^4
  v[14] = cmul(v[14], w6);
  v[7] = cmul(v[7], w3);
  v[11] = cmul(v[11], w6);
  v[15] = cmul(v[15], w9);
  // Level 2: for each k2, a 4-point DFT over n1: v[4 k2 + n1] lives at v[n1 + 4 k2].
  for (int k2 = 0; k2 < 4; ++k2) bfly4<INV>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
  // Output X[k2 + 4 k1] sits at v[4 k2 + k1]: transpose the 4x4 block.
  float2 t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) t[i] = v[i];
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) v[k2 + 4 * k1] = t[4 * k2 + k1];
  }
}

}  // namespace qpb
