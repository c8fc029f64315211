// One tile of a TMA column pass: LINES adjacent columns (stride S > 1) of L
// points, moved as one [L][LINES] box by tensor-map copies. Shared by the
// column-pass kernel (one tile per CTA, column_pass.cu) and the persistent
// iteration kernel (many tiles per CTA, persistent.cu).
//
// The box lands in shared memory swizzled so that the row-order reads are
// free of bank conflicts; a modulus tile's amplitude (stored by the problem
// set-up in the pass's CTA order, line-major) arrives by a bulk copy on the
// same mbarrier. Inside the CTA the lines are held row-style: the T threads of
// a line share one warp (thread t of line l owns elements t + T m), so the
// Stockham exchanges of the register-resident transform (line_fft.cuh) need
// warp barriers only, and the Fourier-error sum is a warp reduction with one
// FP64 atomic per warp. The result goes back through the same box and leaves
// by one tensor-map store.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "bulk_copy.cuh"
#include "line_fft.cuh"
#include "projection.cuh"
#include "reduce.cuh"
#include "storage.cuh"

namespace qpb {

// CTA shape: LINES_ columns of L points, T threads a line, the wave stored as
// WT (float2 or __half2). A box row is LINES_ elements: 64 or 128 bytes of
// complex64, 32 or 64 of fp16 pairs, swizzled with the pattern of that width.
// The register budget is sized for MIN_CTAS resident CTAs per SM
// (registers <= 64K / (NT * MIN_CTAS)): at 8 lines of 256 points, 5 CTAs per
// SM leave the modulus tile 96 registers (it uses 93). The column pass also
// has a 7-per-SM variant of that tile (72 registers, no spills) for launches
// larger than one wave.
template <int L, class WT, int LINES_>
struct ColumnTiling {
  using G = Geometry<L>;
  static constexpr int LINES = LINES_;
  static constexpr int NT = G::T * LINES;
  // (lines of 512 points: 256 threads and a three-stage transform, 2 CTAs per
  // SM at up to 128 registers)
  static constexpr int MIN_CTAS = NT <= 64 ? 12 : (NT <= 128 ? 5 : (L >= 512 ? 2 : 3));
  static constexpr int ROW_BYTES = LINES * static_cast<int>(sizeof(WT));  // one box row
  static constexpr int kBox = L * ROW_BYTES;
  // A tensor-map box is at most 256 rows high: longer lines move in parts of
  // kBoxRows rows, one copy each, to consecutive parts of the box.
  static constexpr int kBoxRows = L < 256 ? L : 256;
  static constexpr int kBoxParts = L / kBoxRows;
  // A half-warp holds 8 threads of each of two lines (column_tile_run); their
  // exchange rows sit 8 mod 16 complex values apart so that the two lines'
  // accesses fall on disjoint banks.
  static constexpr int PITCH = (G::PITCH + 7) / 16 * 16 + 8;
  static constexpr int kExchange = LINES * PITCH * 8;
  // the box, later the lines' exchange rows; a multiple of 1024 bytes
  static constexpr int kRegion = ((kBox > kExchange ? kBox : kExchange) + 1023) / 1024 * 1024;
  static_assert(ROW_BYTES == 128 || ROW_BYTES == 64 || ROW_BYTES == 32,
                "the swizzles below are the 128/64/32-byte patterns");
  static_assert(G::T <= 32 && 32 % G::T == 0, "a line's threads must share one warp");
  static_assert(NT % 32 == 0, "whole warps");
};

template <int L, Mode M, class AmpT, class WT, int LINES>
struct ColumnStaging {
  using Ti = ColumnTiling<L, WT, LINES>;
  static constexpr bool kAmp = M == Mode::kMod;
  static constexpr int kAmpBytes = kAmp ? Ti::LINES * L * static_cast<int>(sizeof(AmpT)) : 0;
  static constexpr int kAmpOffset = Ti::kRegion;
  // the stage-major twiddle table, copied next to the amplitude tile
  static constexpr int kTwBytes = Ti::G::TW_COUNT * 8;
  static constexpr int kTwOffset = kAmpOffset + kAmpBytes;
  static constexpr int kBarrier = (kTwOffset + kTwBytes + 15) / 16 * 16;
  // + 1024: the dynamic shared memory base is aligned up to 1024 bytes inside
  static constexpr int kBytes = kBarrier + 16 + 1024;
  static_assert(kAmpBytes % 16 == 0 && kTwBytes % 16 == 0, "bulk copies need 16-byte sizes");
};

// Byte offset of logical byte `o` of a box in shared memory written with
// CU_TENSOR_MAP_SWIZZLE_128B, _64B or _32B for box rows of that width (the
// 16-byte chunk bits 4-6, 4-5 or 4 XOR address bits 7-9, 7-8 or 7); the box
// starts on a 1024-byte boundary.
template <int ROW_BYTES>
__device__ __forceinline__ int swizzled(int o) {
  constexpr int mask = ROW_BYTES == 128 ? 0x70 : (ROW_BYTES == 64 ? 0x30 : 0x10);
  return o ^ ((o >> 3) & mask);
}

template <int ROW_BYTES>
constexpr CUtensorMapSwizzle swizzle_mode() {
  return ROW_BYTES == 128 ? CU_TENSOR_MAP_SWIZZLE_128B
                          : (ROW_BYTES == 64 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B);
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, std::uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<std::uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int c0, int c1, int c2,
                                             const void* src) {
  asm volatile(
      "cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(
          reinterpret_cast<std::uint64_t>(map)),
      "r"(c0), "r"(c1), "r"(c2), "r"(smem_addr(src))
      : "memory");
}

// Shared memory of one column tile.
struct ColumnSmem {
  unsigned char* box;   // kRegion bytes, 1024-byte aligned
  void* amp;            // kAmpBytes (modulus tiles)
  const float2* tw;     // the stage-major twiddle table (loaded by the caller or the tile)
  std::uint64_t* bar;   // the tile's mbarrier, initialised by the caller
  double** err_slot;    // the modulus tile's error slot (thread 0 writes it)
};

// Tile `tile` of the pass described by `p` (lines tile * LINES ..) in two
// halves. column_tile_issue (thread 0 only) starts the tile's copies on the
// tile's mbarrier and, for a modulus tile, names its error slot: error row
// `err_row` (negative: the row the control block's counter of p.group names).
// With LOAD_TW it also copies the twiddle table to s.tw. column_tile_run (all
// threads) waits for the copies with mbarrier phase `parity`, transforms,
// projects and stores: thread 0 issues and commits the tile's tensor-map
// store, which the caller waits for (its reads before the shared memory is
// reused, its writes before other CTAs read the result). It returns false,
// after waiting once more for copies in flight and counting the failure, when
// the staged wait gave up.
template <int L, Mode M, class AmpT, class WT, int LINES, bool LOAD_TW>
__device__ __forceinline__ void column_tile_issue(const CUtensorMap* wmap, const PassParams& p,
                                                  long long tile, const ColumnSmem& s,
                                                  int err_row) {
  using Ti = ColumnTiling<L, WT, LINES>;
  using St = ColumnStaging<L, M, AmpT, WT, LINES>;
  const long long line0 = tile * LINES;
  const int outer = static_cast<int>(line0 / p.S);
  const int inner0 = static_cast<int>(line0 - static_cast<long long>(outer) * p.S);
  const int batch_start = static_cast<int>(line0 / p.lines_per_start);
  mbar_arrive_expect_tx(s.bar, St::kAmpBytes + (LOAD_TW ? St::kTwBytes : 0) + Ti::kBox);
  if (!p.starve) {
#pragma unroll
    for (int part = 0; part < Ti::kBoxParts; ++part) {
      tma_load_3d(s.box + part * Ti::kBoxRows * Ti::ROW_BYTES, wmap, inner0, part * Ti::kBoxRows,
                  outer, s.bar);
    }
    if constexpr (LOAD_TW) {
      bulk_g2s(const_cast<float2*>(s.tw), p.stage_twiddle, St::kTwBytes, s.bar);
    }
    if constexpr (St::kAmp) {
      const long long line_in_start =
          line0 - static_cast<long long>(batch_start) * p.lines_per_start;
      const AmpT* src = static_cast<const AmpT*>(p.amp) + amp_offset(p, p.start0 + batch_start) +
                        line_in_start * L;
      bulk_g2s(s.amp, src, St::kAmpBytes, s.bar);
    }
  }
  // control values while the copies are in flight: the error row
  if constexpr (M == Mode::kMod) {
    const Ctrl* c = p.ctrl;
    const int r = err_row >= 0 ? err_row : c->counters[p.group];
    *s.err_slot = r < c->capacity
                      ? c->errs + static_cast<long long>(r) * p.starts_total + p.start0 + batch_start
                      : nullptr;
  }
}

template <int L, Mode M, class AmpT, class WT, int LINES>
__device__ __forceinline__ bool column_tile_run(const CUtensorMap* wmap, const PassParams& p,
                                                long long tile, const ColumnSmem& s,
                                                unsigned parity) {
  using G = Geometry<L>;
  using Ti = ColumnTiling<L, WT, LINES>;
  constexpr int E = G::E;
  constexpr int T = G::T;
  const int tid = threadIdx.x;
  // Line l and thread t of the line: with 16 threads a line, a half-warp
  // holds threads t = 8 h .. 8 h + 7 of two lines (lane = 16 h + 8 (l & 1) +
  // t mod 8), so that each 64-bit half-warp access of the swizzled box touches
  // 8 rows of 2 columns, 16 distinct 8-byte slots; shorter lines hold 8
  // threads, already 2 lines a half-warp (lane = 8 (l mod 4) + t).
  const int lane = tid & 31;
  const int l = T == 16 ? (tid >> 5) * 2 + ((lane >> 3) & 1) : tid / T;
  const int t = T == 16 ? (lane >> 4) * 8 + (lane & 7) : tid % T;
  const long long line0 = tile * LINES;
  const int outer = static_cast<int>(line0 / p.S);
  const int inner0 = static_cast<int>(line0 - static_cast<long long>(outer) * p.S);

  if (!__syncthreads_and(mbar_wait(s.bar, parity, p.wait_tries) ? 1 : 0)) {
    if (tid == 0) {
      mbar_wait(s.bar, parity, p.wait_tries);  // copies still in flight land first
      atomicAdd(p.wait_failures, 1);
    }
    return false;
  }

  // Box byte offset of element t + T m of this thread's line: the swizzle
  // repeats every 8 box rows and T is a multiple of 8, so the XOR bits are
  // those of row t and the offset is this thread's one plus m T ROW_BYTES.
  static_assert(T % 8 == 0, "the swizzle pattern must repeat every T rows");
  const int lane_box = swizzled<Ti::ROW_BYTES>(t * Ti::ROW_BYTES + l * static_cast<int>(sizeof(WT)));
  float2 v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    v[m] = load_c(*reinterpret_cast<const WT*>(s.box + lane_box + m * T * Ti::ROW_BYTES));
  }
  __syncthreads();  // the box becomes the lines' exchange rows
  float2* row = reinterpret_cast<float2*>(s.box) + l * Ti::PITCH;

  if constexpr (M == Mode::kMod) {
    transform<L, false, true, true, true>(v, t, s.tw, row);
    // line l of the tile is stored rotated by amp_line_rotation(L, l)
    const AmpT* amp_tile = static_cast<const AmpT*>(s.amp) + l * L;
    const int rot = amp_line_rotation(L, l);
    const float sc = p.scale;
    float acc = 0.0f;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      // an fp16 wave defers the inverse's 1/sqrt(n) to the update pass
      v[m] = pointwise_projection<Mode::kMod>(v[m], to_float(amp_tile[(t + T * m + rot) & (L - 1)]),
                                              sc, acc, kHalfStorage<WT> ? 1.0f : sc);
    }
    // every line of the tile belongs to one start: one atomic per warp
    const double total = warp_sum_double(static_cast<double>(acc));
    if ((tid & 31) == 0) {
      double* slot = *s.err_slot;
      if (slot) atomicAdd(slot, total);
    }
    transform<L, true, true, true, true>(v, t, s.tw, row);
  } else {
    transform<L, M == Mode::kInv, true, true, true>(v, t, s.tw, row);
  }

  __syncthreads();  // every line is done with the exchange rows
#pragma unroll
  for (int m = 0; m < E; ++m) {
    *reinterpret_cast<WT*>(s.box + lane_box + m * T * Ti::ROW_BYTES) = store_c<WT>(v[m]);
  }
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int part = 0; part < Ti::kBoxParts; ++part) {
      tma_store_3d(wmap, inner0, part * Ti::kBoxRows, outer,
                   s.box + part * Ti::kBoxRows * Ti::ROW_BYTES);
    }
    bulk_commit();
  }
  return true;
}

// Both halves, for a CTA that runs one tile.
template <int L, Mode M, class AmpT, class WT, int LINES, bool LOAD_TW>
__device__ __forceinline__ bool column_tile(const CUtensorMap* wmap, const PassParams& p,
                                            long long tile, const ColumnSmem& s, unsigned parity,
                                            int err_row) {
  if (threadIdx.x == 0) column_tile_issue<L, M, AmpT, WT, LINES, LOAD_TW>(wmap, p, tile, s, err_row);
  return column_tile_run<L, M, AmpT, WT, LINES>(wmap, p, tile, s, parity);
}

}  // namespace qpb
