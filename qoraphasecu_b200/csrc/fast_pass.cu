// Streamed line passes for power-of-two line lengths 16..1024: each CTA moves
// a tile of lines from HBM, transforms them with the register-resident
// Stockham transforms of line_fft.cuh, applies the pass's point-wise step and
// writes the tile back.
//
// Rows (stride 1) map 16..256 lines to a CTA, threads of a line adjacent;
// columns (stride S) map adjacent lines to adjacent threads, so a half-warp
// reads 16 neighbouring elements of one row either way (128-byte segments).

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>
#include <stdexcept>

#include "bulk_copy.cuh"
#include "dependent_launch.cuh"
#include "fast_pass.cuh"
#include "line_fft.cuh"
#include "projection.cuh"
#include "reduce.cuh"
#include "storage.cuh"

namespace qpb {

namespace {

__host__ __device__ constexpr int align16(int bytes) { return (bytes + 15) / 16 * 16; }

// Shared-memory layout of one CTA. Region W holds the Stockham exchange rows
// and, for row passes that move whole tiles by bulk copies, the wave tile in
// and out (its rows are contiguous in global memory; rows of 128 points are
// staged kRowPitch elements apart); then the side inputs staged by bulk
// copies (the amplitude tile of a modulus pass; the old-iterate and support
// tiles of a row update); then a row update's copy of the stage-major twiddle
// table; then two mbarriers (16 bytes).
// CTA shape of a streamed pass: lines per CTA, threads, the CTAs per SM the
// register budget is sized for (registers <= 64K / (NT * MIN_CTAS)) and the
// exchange rows. Rows of 256 points use 4 lines per CTA (64 threads, up to 12
// CTAs per SM), which shortens a launch's last partial wave, and rows of 128
// use 8 (64 threads; the 128^3 x-axis update pass measured 60.5 us against
// 69.6 us with 32 lines and 62.6 us with 4). Rows of 512 and 1024 points take
// one line per CTA, budgeted 128 registers a thread (their three-stage
// transforms spill at 80): a 512^2 update pass of 16 starts measured 29.6 us
// against 39.4 us with 16 lines per CTA and 30.8 us with 2. Columns of 128
// points take 16 lines (128 threads; the 128^3 z-axis modulus pass measured
// 42 us against 47 us with 32 lines); other columns keep 256 / T lines up
// to 256 points (16 at 256, and at 512), whose 128-byte and longer row
// segments load better (fewer columns per CTA measured slower: 8 at 512 took
// 37.2 us against 35.2 us, 8 at 128 ran the 128^3 workload 17% slower).
template <int L, bool ROWS>
struct Tiling {
  using G = Geometry<L>;
  static constexpr int LINES = (ROWS && L >= 512)   ? 1
                               : (ROWS && L == 256) ? 4
                               : (ROWS && L == 128) ? 8
                               : (!ROWS && L == 128) ? 16
                                                    : (G::T <= 16 ? 256 / G::T : (L >= 1024 ? 8 : 16));
  static constexpr int NT = G::T * LINES;
  static constexpr int MIN_CTAS = L >= 512 ? (NT < 512 ? 512 / NT : 1)
                                           : (NT <= 64 ? 12 : (NT <= 128 ? 6 : (NT <= 256 ? 3 : 1)));
};

// WT, XT: storage of the wave and of the iterate (float2 or __half2).
template <int L, bool ROWS, Mode M, class AmpT, class WT, class XT>
struct Staging {
  using G = Tiling<L, ROWS>;
  using InT = std::conditional_t<M == Mode::kFwdFromX, XT, WT>;
  static constexpr bool kRowTma =
      ROWS && (M == Mode::kFwd || M == Mode::kFwdFromX || M == Mode::kInv || M == Mode::kUpd);
  static constexpr bool kAmp = M == Mode::kMod || M == Mode::kGrad;
  static constexpr bool kUpd = M == Mode::kUpd && ROWS;
  // Rows of 128 points (8 threads a row, a half-warp holding two rows) sit
  // kRowPitch elements apart in the staged wave, iterate and output tiles, one
  // bulk copy per row, and the exchange rows kXPitch = 8 mod 16 values apart,
  // so that the two rows of a half-warp fall on disjoint banks (rows L apart
  // share them: the 128^3 x-axis update counted 2.3 M conflicts on 5.6 M
  // shared-load wavefronts per launch of 4 starts).
  static constexpr bool kPadRows = kRowTma && G::LINES > 1 && L == 128;
  static constexpr int kRowPitch = kPadRows ? L + 8 : L;
  static constexpr int kXPitch = kPadRows ? (Geometry<L>::PITCH + 7) / 16 * 16 + 8
                                          : Geometry<L>::PITCH;
  static constexpr int kTileIn = G::LINES * L * static_cast<int>(sizeof(InT));
  static constexpr int kTileOut = G::LINES * L * static_cast<int>(sizeof(WT));
  static constexpr int kTileSmem = G::LINES * kRowPitch *
                                   static_cast<int>(sizeof(InT) > sizeof(WT) ? sizeof(InT)
                                                                             : sizeof(WT));
  static constexpr int kRowsSmem = Geometry<L>::STAGES > 1 ? G::LINES * kXPitch * 8 : 0;
  static constexpr int kExchange =
      align16(kRowTma && kTileSmem > kRowsSmem ? kTileSmem : kRowsSmem);
  static constexpr int kSideA = kAmp   ? G::LINES * L * static_cast<int>(sizeof(AmpT))
                                : kUpd ? G::LINES * kRowPitch * static_cast<int>(sizeof(XT))
                                       : 0;
  static constexpr int kSideABytes =  // bytes the side-A copies deliver
      kUpd ? G::LINES * L * static_cast<int>(sizeof(XT)) : kSideA;
  // The support tile's rows of up to 128 points sit L + 16 bytes apart (one
  // bulk copy per row), which puts the 4 rows a warp reads on different banks:
  // the 128^3 x-axis update pass went from 59.0 to 57.3 us. Rows of 256 keep
  // one copy per tile (2 rows a warp, 2-way conflicts): a copy per row cost
  // more there (11.26 -> 11.57 us for 32 starts of 256^2).
  static constexpr int kSupportPitch = G::LINES > 1 && L <= 128 ? L + 16 : L;
  static constexpr int kSupportBytes = G::LINES * L;  // bytes the copies deliver
  static constexpr int kSideB = kUpd ? G::LINES * kSupportPitch : 0;
  static constexpr bool kBarrierUsed = kAmp || kUpd || kRowTma;
  // A row update (two transforms per tile) reads its twiddles from a copy of
  // the stage-major table in shared memory, copied with the wave tile.
  static constexpr bool kTwStaged = kUpd && Geometry<L>::STAGES > 1 && L <= 256;
  static constexpr int kTwOffset = align16(kExchange + kSideA + kSideB);
  static constexpr int kTwBytes = kTwStaged ? Geometry<L>::TW_COUNT * 8 : 0;
  static constexpr int kBarrier = align16(kTwOffset + kTwBytes);
  static constexpr int kBytes = kBarrierUsed ? kBarrier + 16 : kRowsSmem;
  static_assert(kSideA % 16 == 0 && kSideB % 16 == 0 && kTileIn % 16 == 0 && kTileOut % 16 == 0 &&
                    kTwBytes % 16 == 0 && kSideABytes % 16 == 0 && kSupportBytes % 16 == 0,
                "bulk copies need 16-byte sizes");
};

template <int L, bool ROWS, Mode M, class AmpT, class WT, class XT>
__global__ void __launch_bounds__(Tiling<L, ROWS>::NT, Tiling<L, ROWS>::MIN_CTAS)
    fast_pass_kernel(const PassParams p) {
  using G = Geometry<L>;
  using Ti = Tiling<L, ROWS>;
  using St = Staging<L, ROWS, M, AmpT, WT, XT>;
  using InT = typename St::InT;
  constexpr int E = G::E;
  constexpr int T = G::T;
  extern __shared__ float2 smem[];
  const int tid = threadIdx.x;
  const int l = ROWS ? tid / T : tid % Ti::LINES;
  const int t = ROWS ? tid % T : tid / Ti::LINES;
  float2* row = smem + l * St::kXPitch;
  wait_for_prior_kernel();  // its wave, iterate, support and control block
  allow_next_kernel();

  const long long line0 = static_cast<long long>(blockIdx.x) * Ti::LINES;
  const int batch_start = static_cast<int>(line0 / p.lines_per_start);
  const long long start_off = static_cast<long long>(batch_start) * p.n;
  // Element t + T m of line (line0 + l) sits at base + (t + T m) * S; the
  // offsets from the thread's first element fit 32 bits (L * S <= n).
  long long base;
  int step;  // distance between a thread's consecutive elements
  if constexpr (ROWS) {
    base = (line0 + l) * L + t;
    step = T;
  } else {
    const long long outer = line0 / p.S;
    const long long inner = line0 - outer * p.S + l;
    base = outer * static_cast<long long>(L) * p.S + inner + static_cast<long long>(t) * p.S;
    step = T * p.S;
  }
  // Every mode that reads both x and w through these pointers (the column
  // update and blur of |x|, the column forward from x) runs on distinct
  // arrays; an operator that transforms in place (w == x) does so only in
  // modes that reach x or w by bulk copies or through one of them.
  WT* __restrict__ wl = reinterpret_cast<WT*>(p.w) + base;
  XT* __restrict__ xl = reinterpret_cast<XT*>(p.x) + base;
  const float2* __restrict__ tw =
      St::kTwStaged ? reinterpret_cast<const float2*>(reinterpret_cast<unsigned char*>(smem) +
                                                      St::kTwOffset)
                    : p.stage_twiddle;
  constexpr bool kTwShared = St::kTwStaged;
  // A row's T threads share a warp, so its exchanges need warp barriers only.
  constexpr bool kWarpLocal = ROWS && T <= 32;

  // Control values are read before the transform so that their latency hides
  // behind it: the error row (thread 0 of a modulus pass) and the update
  // coefficients.
  [[maybe_unused]] double* err_slot = nullptr;
  if constexpr (M == Mode::kMod || M == Mode::kGrad) {
    if (tid == 0) {
      const Ctrl* c = p.ctrl;
      const int r = c->counters[p.group];
      if (r < c->capacity) {
        err_slot = c->errs + static_cast<long long>(r) * p.starts_total + p.start0 + batch_start;
      }
    }
  }
  [[maybe_unused]] float ca = p.coef_a, cb = p.coef_b;
  if constexpr (M == Mode::kUpd) {
    if (p.coef_from_ctrl) {
      ca = p.ctrl->a;
      cb = p.ctrl->b;
    }
  }

  // Inputs that do not depend on the transform go to shared memory by bulk
  // asynchronous copies issued first: the whole input tile of a row pass, the
  // amplitude tile of a modulus pass, the old iterate and support of a row
  // update. They hold no registers while in flight.
  unsigned char* sbase = reinterpret_cast<unsigned char*>(smem);
  // region W, rows of length L (bulk-copied passes): the input tile, later the output tile
  [[maybe_unused]] const InT* in_tile = reinterpret_cast<const InT*>(smem);
  [[maybe_unused]] WT* out_tile = reinterpret_cast<WT*>(smem);
  // Two barriers: `bar` for the input tile (or the amplitude), `side_bar` for
  // the old iterate and support of a row update, which are needed only after
  // the inverse transform, so their copies overlap it.
  [[maybe_unused]] auto* bar = reinterpret_cast<std::uint64_t*>(sbase + St::kBarrier);
  [[maybe_unused]] std::uint64_t* side_bar = St::kUpd ? bar + 1 : bar;
  if constexpr (St::kBarrierUsed) {
    if (tid == 0) {
      mbar_init(bar, 1);
      if constexpr (St::kUpd) {
        mbar_arrive_expect_tx(bar, St::kTileIn + St::kTwBytes);
        mbar_init(side_bar, 1);
        mbar_arrive_expect_tx(side_bar, St::kSideABytes + St::kSupportBytes);
      } else {
        mbar_arrive_expect_tx(bar, (St::kRowTma ? St::kTileIn : 0) + St::kSideA + St::kSideB);
      }
    }
    __syncthreads();
    // p.starve (tests of the timeout path) leaves every copy out, so the
    // waits below run out with nothing in flight.
    if constexpr (St::kRowTma) {
      if (tid == 0 && !p.starve) {
        const InT* src = reinterpret_cast<const InT*>(M == Mode::kFwdFromX ? p.x : p.w) + line0 * L;
        if constexpr (St::kPadRows) {
          for (int r = 0; r < Ti::LINES; ++r) {
            bulk_g2s(reinterpret_cast<InT*>(smem) + r * St::kRowPitch, src + r * L,
                     L * static_cast<int>(sizeof(InT)), bar);
          }
        } else {
          bulk_g2s(smem, src, St::kTileIn, bar);
        }
        if constexpr (St::kTwStaged) {
          bulk_g2s(sbase + St::kTwOffset, p.stage_twiddle, St::kTwBytes, bar);
        }
      }
    }
    if constexpr (St::kUpd) {
      if (tid == 0 && !p.starve) {
        const XT* xsrc = reinterpret_cast<const XT*>(p.x) + line0 * L;
        if constexpr (St::kPadRows) {
          for (int r = 0; r < Ti::LINES; ++r) {
            bulk_g2s(reinterpret_cast<XT*>(sbase + St::kExchange) + r * St::kRowPitch,
                     xsrc + r * L, L * static_cast<int>(sizeof(XT)), side_bar);
          }
        } else {
          bulk_g2s(sbase + St::kExchange, xsrc, St::kSideA, side_bar);
        }
        if constexpr (St::kSupportPitch == L) {
          bulk_g2s(sbase + St::kExchange + St::kSideA, p.support + line0 * L, St::kSupportBytes,
                   side_bar);
        } else {
          for (int r = 0; r < Ti::LINES; ++r) {
            bulk_g2s(sbase + St::kExchange + St::kSideA + r * St::kSupportPitch,
                     p.support + (line0 + r) * L, L, side_bar);
          }
        }
      }
    } else if constexpr (St::kAmp) {
      if (ROWS || p.amp_tiled) {
        // FFT-order rows, or the amplitude pre-tiled in this pass's CTA order:
        // the CTA's tile is one contiguous block.
        if (tid == 0 && !p.starve) {
          const long long line_in_start =
              line0 - static_cast<long long>(batch_start) * p.lines_per_start;
          const AmpT* src = static_cast<const AmpT*>(p.amp) +
                            amp_offset(p, p.start0 + batch_start) + line_in_start * L;
          bulk_g2s(sbase + St::kExchange, src, St::kSideA, bar);
        }
      } else {
        // one copy per element index j of the lines: LINES adjacent amplitudes
        const long long outer = line0 / p.S;
        const AmpT* src = static_cast<const AmpT*>(p.amp) + amp_offset(p, p.start0 + batch_start) +
                          (outer * static_cast<long long>(L) * p.S + (line0 - outer * p.S) - start_off);
        constexpr int kRowBytes = Ti::LINES * static_cast<int>(sizeof(AmpT));
        for (int j = tid; j < L && !p.starve; j += Ti::NT) {
          bulk_g2s(sbase + St::kExchange + j * kRowBytes, src + static_cast<long long>(j) * p.S,
                   kRowBytes, bar);
        }
      }
    }
  }

  // Every thread waits (bounded); if any gave up, the CTA leaves together,
  // writing nothing. Before it leaves, thread 0 waits once more (bounded
  // again) on every barrier whose copies may still be in flight, so that no
  // copy lands in the shared memory of a CTA that has exited, and records the
  // failure in the launching owner's counter.
  auto staged = [&](std::uint64_t* b) -> bool {
    if (!__syncthreads_and(mbar_wait(b, 0, p.wait_tries) ? 1 : 0)) {
      if (tid == 0) {
        mbar_wait(bar, 0, p.wait_tries);
        if constexpr (St::kUpd) mbar_wait(side_bar, 0, p.wait_tries);
        atomicAdd(p.wait_failures, 1);
      }
      return false;
    }
    return true;
  };

  float2 v[E];
  if constexpr (St::kRowTma) {
    if (!staged(bar)) return;
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = load_c(in_tile[l * St::kRowPitch + t + T * m]);
    __syncthreads();  // region W becomes the exchange buffer
  } else {
#pragma unroll
    for (int m = 0; m < E; ++m) {
      if constexpr (M == Mode::kFwdFromX) {
        v[m] = load_c(xl[m * step]);
      } else if constexpr (M == Mode::kBlurMag) {
        const float2 xv = load_c(xl[m * step]);
        v[m] = {sqrtf(xv.x * xv.x + xv.y * xv.y), 0.0f};
      } else {
        v[m] = load_c(wl[m * step]);
      }
    }
  }

  constexpr bool kStartsInverse = M == Mode::kInv || M == Mode::kUpd;
  // The last exchange's closing barrier is needed only before a second
  // transform with no block barrier in between (the blur's); a modulus pass
  // passes one in its error sum, an update in its store, and the passes of a
  // single transform only write the row again after the barrier below.
  constexpr bool kTrail = M == Mode::kBlur || M == Mode::kBlurMag;
  transform<L, kStartsInverse, kWarpLocal, kTrail, kTwShared>(v, t, tw, row);

  if constexpr (St::kAmp) {
    if (!staged(bar)) return;
  }

  if constexpr (M == Mode::kMod || M == Mode::kGrad) {
    const float s = p.scale;
    float acc = 0.0f;
    const AmpT* amp_tile = reinterpret_cast<const AmpT*>(sbase + St::kExchange);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int j = t + T * m;
      const float a = to_float(ROWS ? amp_tile[l * L + j] : amp_tile[j * Ti::LINES + l]);
      // an fp16 wave defers the inverse's 1/sqrt(n) to the update pass
      v[m] = pointwise_projection<M>(v[m], a, s, acc, kHalfStorage<WT> ? 1.0f : s);
    }
    // one call per CTA; its first barrier also orders the forward transform's
    // exchange reads before the inverse's writes
    const double total = block_sum_double<false>(static_cast<double>(acc));
    if (tid == 0 && err_slot) atomicAdd(err_slot, total);
    transform<L, true, kWarpLocal, false, kTwShared>(v, t, tw, row);
  } else if constexpr (M == Mode::kUpd) {
    if constexpr (St::kUpd) {
      if (!staged(side_bar)) return;
      // x_new replaces the old iterate in its tile and leaves by one bulk store.
      XT* x_tile = reinterpret_cast<XT*>(sbase + St::kExchange);
      const std::uint8_t* s_tile = sbase + St::kExchange + St::kSideA;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        const int j = l * St::kRowPitch + t + T * m;
        float2 xn = kHalfStorage<WT> ? cscale(v[m], p.scale) : v[m];
        if (!s_tile[l * St::kSupportPitch + t + T * m]) {
          const float2 xo = load_c(x_tile[j]);
          xn = {ca * xo.x + cb * xn.x, ca * xo.y + cb * xn.y};
        }
        x_tile[j] = store_c<XT>(xn);
        v[m] = xn;
      }
      fence_proxy_async();
      __syncthreads();
      if (tid == 0) {
        XT* xdst = reinterpret_cast<XT*>(p.x) + line0 * L;
        if constexpr (St::kPadRows) {
          for (int r = 0; r < Ti::LINES; ++r) {
            bulk_s2g(xdst + r * L, x_tile + r * St::kRowPitch, L * static_cast<int>(sizeof(XT)));
          }
        } else {
          bulk_s2g(xdst, x_tile, St::kSideA);
        }
        bulk_commit();
      }
    } else {
      const std::uint8_t* __restrict__ sl = p.support + base;
#pragma unroll
      for (int m = 0; m < E; ++m) {
        float2 xn = kHalfStorage<WT> ? cscale(v[m], p.scale) : v[m];
        if (!sl[m * step]) {
          const float2 xo = load_c(xl[m * step]);
          xn = {ca * xo.x + cb * xn.x, ca * xo.y + cb * xn.y};
        }
        xl[m * step] = store_c<XT>(xn);
        v[m] = xn;
      }
      __syncthreads();
    }
    if (p.bump_counter && blockIdx.x == 0 && tid == 0) ++p.ctrl->counters[p.group];
    transform<L, false, kWarpLocal, false, kTwShared>(v, t, tw, row);
  } else if constexpr (M == Mode::kBlur || M == Mode::kBlurMag) {
    const float inv_l = 1.0f / static_cast<float>(L);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int j = t + T * m;
      const float f = fftfreq(static_cast<std::uint32_t>(j), static_cast<std::uint32_t>(L));
      v[m] = cscale(v[m], expf(p.blur_k * f * f) * inv_l);
    }
    transform<L, true, kWarpLocal, false>(v, t, tw, row);
  }

  if constexpr (St::kRowTma) {
    // Region W is free once every warp is past its last exchange: the output
    // tile goes there and leaves by one bulk store.
    __syncthreads();
#pragma unroll
    for (int m = 0; m < E; ++m) out_tile[l * St::kRowPitch + t + T * m] = store_c<WT>(v[m]);
    fence_proxy_async();
    __syncthreads();
    if (tid == 0) {
      WT* wdst = reinterpret_cast<WT*>(p.w) + line0 * L;
      if constexpr (St::kPadRows) {
        for (int r = 0; r < Ti::LINES; ++r) {
          bulk_s2g(wdst + r * L, out_tile + r * St::kRowPitch, L * static_cast<int>(sizeof(WT)));
        }
      } else {
        bulk_s2g(wdst, out_tile, St::kTileOut);
      }
      bulk_commit();
      bulk_wait_reads();
    }
    return;
  }

  float peak = 0.0f;
  float sq = 0.0f;
  unsigned cnt = 0;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    wl[m * step] = store_c<WT>(v[m]);
    if constexpr (M == Mode::kBlur || M == Mode::kBlurMag) {
      if (p.level_method == 1) {
        peak = fmaxf(peak, v[m].x);
      } else if (p.level_method == 2 && p.support[base + m * step]) {
        sq += v[m].x * v[m].x;
        ++cnt;
      }
    }
  }
  if constexpr (M == Mode::kBlur || M == Mode::kBlurMag) {
    if (p.level_method == 1) {
      peak = warp_max(peak);
      if ((tid & 31) == 0) atomicMax(&p.level[batch_start].max_bits, __float_as_int(peak));
    } else if (p.level_method == 2) {
      const double s2 = block_sum_double(static_cast<double>(sq));
      __syncthreads();
      const double c2 = block_sum_double(static_cast<double>(cnt));
      if (tid == 0) {
        atomicAdd(&p.level[batch_start].sum, s2);
        atomicAdd(&p.level[batch_start].count, static_cast<unsigned long long>(c2));
      }
    }
  }
}

template <int L, bool ROWS, Mode M, class AmpT, class WT, class XT>
void launch_one(const PassParams& p, cudaStream_t stream) {
  using Ti = Tiling<L, ROWS>;
  const dim3 grid(static_cast<unsigned>(p.lines / Ti::LINES));
  launch_dependent(fast_pass_kernel<L, ROWS, M, AmpT, WT, XT>, grid, dim3(Ti::NT),
                   Staging<L, ROWS, M, AmpT, WT, XT>::kBytes, stream, p);
  count_launches(1);
}

// Storage combinations built: complex64 wave and iterate for every mode; an
// fp16 wave with an fp16 or complex64 iterate for the modes of an iteration
// and of the wave's set-up (FP32 amplitude); the blur of an fp16 iterate into
// a complex64 wave (shrinkwrap). Modes that do not touch x use one kernel for
// either iterate storage.
template <Mode M>
inline constexpr bool kHalfWaveMode = M == Mode::kFwd || M == Mode::kFwdFromX ||
                                      M == Mode::kInv || M == Mode::kMod || M == Mode::kUpd;
template <Mode M>
inline constexpr bool kTouchesX = M == Mode::kFwdFromX || M == Mode::kUpd || M == Mode::kBlurMag;

template <int L, bool ROWS, Mode M>
void launch_storage(const PassParams& p, cudaStream_t stream) {
  if (p.wave_half || (kTouchesX<M> && p.iter_half)) {
    if (p.amp_storage != AmpStorage::kF32) {
      throw std::logic_error("fast line pass: fp16 storage runs with an FP32 amplitude");
    }
    if constexpr (kHalfWaveMode<M>) {
      if (p.wave_half) {
        if (p.iter_half || !kTouchesX<M>) {
          return launch_one<L, ROWS, M, float, __half2, __half2>(p, stream);
        }
        return launch_one<L, ROWS, M, float, __half2, float2>(p, stream);
      }
    }
    if constexpr (M == Mode::kBlurMag) {
      if (!p.wave_half) return launch_one<L, ROWS, M, float, float2, __half2>(p, stream);
    }
    throw std::logic_error("fast line pass: no kernel for this storage and mode");
  }
  if constexpr (M == Mode::kMod || M == Mode::kGrad) {
    switch (p.amp_storage) {
      case AmpStorage::kF32:
        return launch_one<L, ROWS, M, float, float2, float2>(p, stream);
      case AmpStorage::kF16:
        return launch_one<L, ROWS, M, __half, float2, float2>(p, stream);
      case AmpStorage::kBF16:
        return launch_one<L, ROWS, M, __nv_bfloat16, float2, float2>(p, stream);
    }
  } else {
    launch_one<L, ROWS, M, float, float2, float2>(p, stream);
  }
}

template <int L, bool ROWS>
void launch_mode(Mode mode, const PassParams& p, cudaStream_t stream) {
  switch (mode) {
    case Mode::kFwd:
      return launch_storage<L, ROWS, Mode::kFwd>(p, stream);
    case Mode::kFwdFromX:
      return launch_storage<L, ROWS, Mode::kFwdFromX>(p, stream);
    case Mode::kInv:
      return launch_storage<L, ROWS, Mode::kInv>(p, stream);
    case Mode::kMod:
      return launch_storage<L, ROWS, Mode::kMod>(p, stream);
    case Mode::kUpd:
      return launch_storage<L, ROWS, Mode::kUpd>(p, stream);
    case Mode::kBlur:
      return launch_storage<L, ROWS, Mode::kBlur>(p, stream);
    case Mode::kBlurMag:
      return launch_storage<L, ROWS, Mode::kBlurMag>(p, stream);
    case Mode::kGrad:
      return launch_storage<L, ROWS, Mode::kGrad>(p, stream);
  }
}

template <int L>
void launch_length(Mode mode, const PassParams& p, cudaStream_t stream) {
  if (p.S == 1) {
    launch_mode<L, true>(mode, p, stream);
  } else {
    launch_mode<L, false>(mode, p, stream);
  }
}

template <int L>
int lines_per_cta(bool rows) {
  return rows ? Tiling<L, true>::LINES : Tiling<L, false>::LINES;
}

}  // namespace

StageGeometry stage_geometry(int L) {
  switch (L) {
    case 16: return stage_geometry_of<16>();
    case 32: return stage_geometry_of<32>();
    case 64: return stage_geometry_of<64>();
    case 128: return stage_geometry_of<128>();
    case 256: return stage_geometry_of<256>();
    case 512: return stage_geometry_of<512>();
    case 1024: return stage_geometry_of<1024>();
    default: return {};
  }
}

namespace {

int fast_lines(int L, bool rows) {
  switch (L) {
    case 16: return lines_per_cta<16>(rows);
    case 32: return lines_per_cta<32>(rows);
    case 64: return lines_per_cta<64>(rows);
    case 128: return lines_per_cta<128>(rows);
    case 256: return lines_per_cta<256>(rows);
    case 512: return lines_per_cta<512>(rows);
    case 1024: return lines_per_cta<1024>(rows);
    default: return 0;
  }
}

template <int L, bool ROWS, Mode M, class AmpT, class WT = float2, class XT = float2>
void allow_smem_one() {
  constexpr int bytes = Staging<L, ROWS, M, AmpT, WT, XT>::kBytes;
  if constexpr (bytes > 48 * 1024) {
    QPB_CHECK(cudaFuncSetAttribute(fast_pass_kernel<L, ROWS, M, AmpT, WT, XT>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  }
}

template <int L, bool ROWS, Mode M>
void allow_smem_half() {
  allow_smem_one<L, ROWS, M, float, __half2, __half2>();
  if constexpr (kTouchesX<M>) allow_smem_one<L, ROWS, M, float, __half2, float2>();
}

template <int L, bool ROWS>
void allow_smem_modes() {
  allow_smem_one<L, ROWS, Mode::kFwd, float>();
  allow_smem_one<L, ROWS, Mode::kFwdFromX, float>();
  allow_smem_one<L, ROWS, Mode::kInv, float>();
  allow_smem_one<L, ROWS, Mode::kMod, float>();
  allow_smem_one<L, ROWS, Mode::kMod, __half>();
  allow_smem_one<L, ROWS, Mode::kMod, __nv_bfloat16>();
  allow_smem_one<L, ROWS, Mode::kUpd, float>();
  allow_smem_one<L, ROWS, Mode::kBlur, float>();
  allow_smem_one<L, ROWS, Mode::kBlurMag, float>();
  allow_smem_one<L, ROWS, Mode::kGrad, float>();
  allow_smem_one<L, ROWS, Mode::kGrad, __half>();
  allow_smem_one<L, ROWS, Mode::kGrad, __nv_bfloat16>();
  allow_smem_half<L, ROWS, Mode::kFwd>();
  allow_smem_half<L, ROWS, Mode::kFwdFromX>();
  allow_smem_half<L, ROWS, Mode::kInv>();
  allow_smem_half<L, ROWS, Mode::kMod>();
  allow_smem_half<L, ROWS, Mode::kUpd>();
  allow_smem_one<L, ROWS, Mode::kBlurMag, float, float2, __half2>();
}

template <int L>
void allow_smem_length() {
  allow_smem_modes<L, true>();
  allow_smem_modes<L, false>();
}

}  // namespace

void configure_fast_passes() {
  static std::mutex mutex;
  static std::set<int> done;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  if (!done.insert(device).second) return;
  allow_smem_length<16>();
  allow_smem_length<32>();
  allow_smem_length<64>();
  allow_smem_length<128>();
  allow_smem_length<256>();
  allow_smem_length<512>();
  allow_smem_length<1024>();
}

bool fast_passes_enabled() {
  static const bool enabled = [] {
    const char* v = std::getenv("QPB_GENERIC_PASSES");
    return !(v && *v && *v != '0');
  }();
  return enabled;
}

int fast_pass_lines(const PassParams& p) {
  return fast_passes_enabled() && fast_pass_supports(p) ? fast_lines(p.L, p.S == 1) : 0;
}

bool fast_pass_supports(const PassParams& p) {
  const int lines = fast_lines(p.L, p.S == 1);
  if (lines == 0) return false;
  if (p.lines_per_start % lines != 0 || p.lines % lines != 0) return false;
  // Columns: the CTA's lines must be adjacent within one outer slab.
  if (p.S != 1 && p.S % lines != 0) return false;
  return true;
}

void launch_fast_pass(Mode mode, const PassParams& p, cudaStream_t stream) {
  switch (p.L) {
    case 16: return launch_length<16>(mode, p, stream);
    case 32: return launch_length<32>(mode, p, stream);
    case 64: return launch_length<64>(mode, p, stream);
    case 128: return launch_length<128>(mode, p, stream);
    case 256: return launch_length<256>(mode, p, stream);
    case 512: return launch_length<512>(mode, p, stream);
    case 1024: return launch_length<1024>(mode, p, stream);
    default: throw std::logic_error("fast line pass: unsupported length");
  }
}

}  // namespace qpb
