// Register-resident Stockham transforms of lines of length L = 16..1024 (powers
// of two), shared by the streamed line passes and the resident iteration kernel.
//
// A line is held by T = L / E threads, E complex values each, in the
// "stride-T" distribution: thread t owns elements t + T m, m < E. Every stage
// of radix R (<= E) is E / R butterflies per thread on registers; between
// stages the values go once through a shared-memory row (written at their
// Stockham output positions, read back in the stride-T distribution). The last
// stage's outputs already sit in the stride-T distribution, so a 256-point
// transform (16 x 16) costs one shared-memory round trip and an inverse
// transform can start from the forward's registers. Rows are padded (one slot
// per 16, pitch = 1 mod 16) so that the Stockham writes and the stride-T reads
// are free of bank conflicts.
#pragma once

#include <cuda_runtime.h>

#include "butterfly.cuh"
#include "common.cuh"
#include "stage_table.hpp"

namespace qpb {

__host__ __device__ constexpr int swz(int i) { return i + (i >> 4); }

template <int L>
struct Geometry {
  static constexpr int E = L == 32 || L == 64 ? 8 : 16;
  static constexpr int T = L / E;
  // Radix of each stage (product = L, each <= E).
  static constexpr int R0 = L <= 16 ? L : E;
  static constexpr int R1 = L <= 16 ? 1 : (L / R0 <= E ? L / R0 : E);
  static constexpr int R2 = L / (R0 * R1);
  static constexpr int STAGES = L <= 16 ? 1 : (R2 == 1 ? 2 : 3);
  static constexpr int PITCH = swz(L) + 1;
  // Offsets of stages 1 and 2 in the stage-major twiddle table, and its size.
  static constexpr int OFF1 = 0;
  static constexpr int OFF2 = (R1 - 1) * R0;
  static constexpr int TW_COUNT = (STAGES >= 2 ? (R1 - 1) * R0 : 0) +
                                  (STAGES >= 3 ? (R2 - 1) * R0 * R1 : 0);
  static_assert(R0 * R1 * R2 == L, "bad factorisation");
  static_assert(R2 <= E && R1 <= E, "radix above the register count");
};

template <int R, bool INV>
__device__ __forceinline__ void butterfly(float2* u) {
  if constexpr (R == 2) {
    bfly2<INV>(u[0], u[1]);
  } else if constexpr (R == 4) {
    bfly4<INV>(u[0], u[1], u[2], u[3]);
  } else if constexpr (R == 8) {
    bfly8<INV>(u);
  } else if constexpr (R == 16) {
    bfly16<INV>(u);
  }
}

// Orders a line's exchange: a block barrier, or a warp barrier when the
// line's T threads share one warp (WARP_LOCAL) and no other warp uses its row.
template <bool WARP_LOCAL>
__device__ __forceinline__ void line_sync() {
  if constexpr (WARP_LOCAL) {
    __syncwarp();
  } else {
    __syncthreads();
  }
}

// One Stockham stage of radix R over the thread's E registers. NS is the
// product of the radices before it; LAST stages leave values in place,
// others exchange through the line's shared-memory row. TRAIL orders the
// exchange's reads before any later write of the row; a caller may drop it
// when a block barrier separates them anyway.
//
// `tw` is the stage-major twiddle table (stage_twiddle_exponent): this
// stage's W_L^{r k L/(NS R)} sits at tw[OFF + (r - 1) NS + k], so the
// threads of a line, whose k are consecutive, read consecutive entries.
// TW_SHARED: the table is a copy in shared memory (plain loads) instead of
// global memory (read-only cached loads).
template <int L, int R, int NS, int OFF, bool LAST, bool INV, bool WARP_LOCAL = false,
          bool TRAIL = true, bool TW_SHARED = false>
__device__ __forceinline__ void stage(float2 (&v)[Geometry<L>::E], int t,
                                      const float2* __restrict__ tw, float2* row) {
  using G = Geometry<L>;
  constexpr int E = G::E;
  constexpr int T = G::T;
  constexpr int Q = E / R;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    float2 u[R];
#pragma unroll
    for (int r = 0; r < R; ++r) u[r] = v[q + r * Q];
    const int j = t + T * q;
    const int k = j & (NS - 1);
    if constexpr (NS > 1) {
#pragma unroll
      for (int r = 1; r < R; ++r) {
        const float2 w = TW_SHARED ? tw[OFF + (r - 1) * NS + k] : __ldg(tw + OFF + (r - 1) * NS + k);
        u[r] = INV ? cmulc(u[r], w) : cmul(u[r], w);
      }
    }
    butterfly<R, INV>(u);
    if constexpr (LAST) {
#pragma unroll
      for (int r = 0; r < R; ++r) v[q + r * Q] = u[r];
    } else {
      const int base = (j - k) * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) row[swz(base + r * NS)] = u[r];
    }
  }
  if constexpr (!LAST) {
    line_sync<WARP_LOCAL>();
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = row[swz(t + T * m)];
    if constexpr (TRAIL) line_sync<WARP_LOCAL>();
  }
}

// Forward (INV false) or inverse unnormalised transform of the line held in
// v. With WARP_LOCAL the caller guarantees that the line's threads share a
// warp (T <= 32, lines not straddling warps) and that no other warp touches
// `row` during the call; then only warp barriers separate the stages. With
// TRAIL false the transform returns without the barrier after its last
// exchange: the caller must pass a block barrier before anything writes the
// row again.
template <int L, bool INV, bool WARP_LOCAL = false, bool TRAIL = true, bool TW_SHARED = false>
__device__ __forceinline__ void transform(float2 (&v)[Geometry<L>::E], int t,
                                          const float2* __restrict__ tw, float2* row) {
  using G = Geometry<L>;
  static_assert(!WARP_LOCAL || G::T <= 32, "a line spans several warps");
  if constexpr (G::STAGES == 1) {
    stage<L, G::R0, 1, 0, true, INV, WARP_LOCAL, true, TW_SHARED>(v, t, tw, row);
  } else if constexpr (G::STAGES == 2) {
    stage<L, G::R0, 1, 0, false, INV, WARP_LOCAL, TRAIL, TW_SHARED>(v, t, tw, row);
    stage<L, G::R1, G::R0, G::OFF1, true, INV, WARP_LOCAL, true, TW_SHARED>(v, t, tw, row);
  } else {
    stage<L, G::R0, 1, 0, false, INV, WARP_LOCAL, true, TW_SHARED>(v, t, tw, row);
    stage<L, G::R1, G::R0, G::OFF1, false, INV, WARP_LOCAL, TRAIL, TW_SHARED>(v, t, tw, row);
    stage<L, G::R2, G::R0 * G::R1, G::OFF2, true, INV, WARP_LOCAL, true, TW_SHARED>(v, t, tw, row);
  }
}

template <int L>
constexpr StageGeometry stage_geometry_of() {
  using G = Geometry<L>;
  StageGeometry g;
  g.stages = G::STAGES;
  g.radix[0] = G::R0;
  g.radix[1] = G::R1;
  g.radix[2] = G::R2;
  g.count = (G::STAGES >= 2 ? (G::R1 - 1) * G::R0 : 0) +
            (G::STAGES >= 3 ? (G::R2 - 1) * G::R0 * G::R1 : 0);
  return g;
}

}  // namespace qpb
