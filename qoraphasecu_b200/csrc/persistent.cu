// The persistent schedule: a chunk of iterations of every start of a 2D
// solver as one kernel launch that walks a work list.
//
// The work list holds, iteration by iteration, the modulus tiles of every
// start (8 adjacent columns each: forward transform along y, modulus
// projection and Fourier-error sum, inverse along y; column_tile.cuh), then
// the update tiles of every start (ROWS adjacent rows each: inverse along x,
// x <- S ? P : a x + b P, forward along x of the new iterate). A CTA claims
// the next item with one atomic, waits until the item's inputs are complete,
// runs it and counts it done:
//   - the modulus tiles of start s in iteration i need all update tiles of
//     start s in iteration i - 1;
//   - the update tiles of start s in iteration i need all its modulus tiles
//     of iteration i.
// Every item depends on items earlier in the list only, and a CTA claims an
// item only while it is running and keeps running until the item is done, so
// every wait ends: the items an item waits for belong to CTAs that are
// running. Start s's update tiles can start while later starts' modulus
// tiles still run, so the two passes of an iteration overlap across starts
// with no launch boundary, and the dynamic claim spreads the work evenly over
// the SMs. Every wait is bounded: a CTA that gives up raises an abort flag
// that the others see, counts the failure in p.wait_failures and leaves, and
// the host turns that into QPB_TIMEOUT.
//
// The tiles publish their results with bulk and tensor-map stores: the
// issuing thread waits for the stores' completion and orders them before the
// release of the counter (proxy fence, GPU-scope fence); a waiting CTA reads
// the counter with acquire semantics and orders its later bulk and
// tensor-map loads after it (proxy fence).

#include <cuda.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <set>
#include <stdexcept>

#include "column_pass.cuh"
#include "column_tile.cuh"
#include "persistent.cuh"

namespace qpb {

namespace {

constexpr int kColumnLines = 8;

template <int LY, int LX>
struct Persist {
  using CT = ColumnTiling<LY, float2, kColumnLines>;
  using CS = ColumnStaging<LY, Mode::kMod, float, float2, kColumnLines>;
  using GX = Geometry<LX>;
  static constexpr int NT = CT::NT;
  static constexpr int ROWS = NT / GX::T;  // rows of one update tile
  static constexpr int MIN_CTAS = NT <= 64 ? 12 : 6;
  // update tile: the wave tile (later its lines' exchange rows), the old
  // iterate, the support
  static constexpr int kRowTile = ROWS * LX * 8;
  static constexpr int kRowExchange = ROWS * GX::PITCH * 8;
  static constexpr int kRowW = ((kRowTile > kRowExchange ? kRowTile : kRowExchange) + 15) / 16 * 16;
  static constexpr int kRowX = kRowTile;
  static constexpr int kRowS = ROWS * LX;
  static constexpr int kRowBytes = kRowW + kRowX + kRowS;
  // modulus tile: the box region and the amplitude tile
  static constexpr int kColBytes = CT::kRegion + CS::kAmpBytes;
  static constexpr int kUnion = ((kColBytes > kRowBytes ? kColBytes : kRowBytes) + 15) / 16 * 16;
  static constexpr int kTwY = LY > 16 ? Geometry<LY>::TW_COUNT * 8 : 0;
  static constexpr int kTwX = LX > 16 ? GX::TW_COUNT * 8 : 0;
  static constexpr int kTwYOffset = kUnion;
  static constexpr int kTwXOffset = kTwYOffset + kTwY;
  static constexpr int kBars = (kTwXOffset + kTwX + 15) / 16 * 16;  // 4 mbarriers
  static constexpr int kSlots = kBars + 32;                         // error slot, item, flag
  static constexpr int kBytes = kSlots + 16 + 1024;                 // + 1024 for alignment
  static_assert(NT % GX::T == 0 && ROWS >= 1, "an update tile is whole rows");
  static_assert(GX::T <= 32 && 32 % GX::T == 0, "a row's threads share one warp");
  static_assert(kRowTile % 16 == 0 && kRowS % 16 == 0 && kTwY % 16 == 0 && kTwX % 16 == 0,
                "bulk copies need 16-byte sizes");
};

__device__ __forceinline__ unsigned load_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Orders this thread's earlier generic-proxy accesses (an acquire) before its
// later asynchronous-proxy global accesses, and the completed bulk stores it
// waited for before its later generic accesses (the release).
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_writes() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

// Polls `counter` until it reaches `target` (at most `tries` polls, each
// after a short sleep) or the abort flag is raised; true when reached.
__device__ bool wait_count(const unsigned* counter, unsigned target, const unsigned* abort,
                           int tries) {
  for (int i = 0; i < tries; ++i) {
    if (load_acquire(counter) >= target) return true;
    if (load_acquire(abort)) return false;
    __nanosleep(64);
  }
  return false;
}

// One update tile: rows tile * ROWS .. of the launch, in shared memory at
// `w_tile` (the wave rows, then the exchange rows, then the output rows),
// `x_tile`, `s_tile`. Bulk stores of x and w are committed by thread 0.
template <int LX, int ROWS>
__device__ __forceinline__ bool update_tile(const PassParams& p, long long tile, float2* w_tile,
                                            float2* x_tile, std::uint8_t* s_tile,
                                            const float2* tw, std::uint64_t* bar,
                                            std::uint64_t* side_bar, unsigned parity, float ca,
                                            float cb) {
  using G = Geometry<LX>;
  constexpr int E = G::E;
  constexpr int T = G::T;
  constexpr unsigned kTile = ROWS * LX * 8;
  const int tid = threadIdx.x;
  const int l = tid / T;
  const int t = tid % T;
  const long long line0 = tile * ROWS;
  if (tid == 0) {
    mbar_arrive_expect_tx(bar, kTile);
    mbar_arrive_expect_tx(side_bar, kTile + ROWS * LX);
    if (!p.starve) {
      bulk_g2s(w_tile, p.w + line0 * LX, kTile, bar);
      bulk_g2s(x_tile, p.x + line0 * LX, kTile, side_bar);
      bulk_g2s(s_tile, p.support + line0 * LX, ROWS * LX, side_bar);
    }
  }
  auto staged = [&](std::uint64_t* b) -> bool {
    if (!__syncthreads_and(mbar_wait(b, parity, p.wait_tries) ? 1 : 0)) {
      if (tid == 0) {
        // copies still in flight land first
        mbar_wait(bar, parity, p.wait_tries);
        mbar_wait(side_bar, parity, p.wait_tries);
        atomicAdd(p.wait_failures, 1);
      }
      return false;
    }
    return true;
  };
  if (!staged(bar)) return false;
  float2 v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) v[m] = w_tile[l * LX + t + T * m];
  __syncthreads();  // the wave rows become the exchange rows
  float2* row = w_tile + l * G::PITCH;
  transform<LX, true, true, true, true>(v, t, tw, row);
  if (!staged(side_bar)) return false;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int j = l * LX + t + T * m;
    float2 xn = v[m];
    if (!s_tile[j]) {
      const float2 xo = x_tile[j];
      xn = {ca * xo.x + cb * xn.x, ca * xo.y + cb * xn.y};
    }
    x_tile[j] = xn;
    v[m] = xn;
  }
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    bulk_s2g(p.x + line0 * LX, x_tile, kTile);
    bulk_commit();
  }
  transform<LX, false, true, true, true>(v, t, tw, row);
  __syncthreads();  // every row is done with the exchange rows
#pragma unroll
  for (int m = 0; m < E; ++m) w_tile[l * LX + t + T * m] = v[m];
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    bulk_s2g(p.w + line0 * LX, w_tile, kTile);
    bulk_commit();
  }
  return true;
}

struct WorkList {
  int starts;
  int iterations;
  int tiles_c;  // modulus tiles per start
  int tiles_r;  // update tiles per start
  unsigned* work;
};

template <int LY, int LX>
__global__ void __launch_bounds__(Persist<LY, LX>::NT, Persist<LY, LX>::MIN_CTAS)
    persistent_kernel(const __grid_constant__ CUtensorMap wmap, const PassParams mod,
                      const PassParams upd, const WorkList wl) {
  using P = Persist<LY, LX>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sbase = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<std::uintptr_t>(smem_raw) + 1023) & ~static_cast<std::uintptr_t>(1023));
  auto* bars = reinterpret_cast<std::uint64_t*>(sbase + P::kBars);
  std::uint64_t* bar_c = bars;      // modulus tiles
  std::uint64_t* bar_w = bars + 1;  // update tiles: the wave rows
  std::uint64_t* bar_s = bars + 2;  // update tiles: old iterate and support
  std::uint64_t* bar_t = bars + 3;  // the twiddle tables, once
  auto* err_slot = reinterpret_cast<double**>(sbase + P::kSlots);
  auto* item_slot = reinterpret_cast<unsigned*>(sbase + P::kSlots + 8);
  auto* flag_slot = reinterpret_cast<int*>(sbase + P::kSlots + 12);
  auto* tw_y = reinterpret_cast<float2*>(sbase + P::kTwYOffset);
  auto* tw_x = reinterpret_cast<float2*>(sbase + P::kTwXOffset);
  unsigned* queue = wl.work;
  unsigned* finished = wl.work + 1;
  unsigned* abort = wl.work + 2;
  unsigned* done_c = wl.work + kPersistentHead;
  unsigned* done_r = done_c + wl.starts;
  const int tid = threadIdx.x;
  const unsigned per_iteration = static_cast<unsigned>(wl.starts) * (wl.tiles_c + wl.tiles_r);
  const unsigned total = per_iteration * static_cast<unsigned>(wl.iterations);

  // The error row of the chunk's first iteration and the update coefficients
  // (the control block does not change during the launch; the counter is read
  // before this CTA claims anything, so before the launch advances it).
  const int row0 = mod.ctrl->counters[mod.group];
  const float ca = upd.coef_from_ctrl ? upd.ctrl->a : upd.coef_a;
  const float cb = upd.coef_from_ctrl ? upd.ctrl->b : upd.coef_b;

  if (tid == 0) {
    for (int b = 0; b < 4; ++b) mbar_init(bars + b, 1);
    mbar_arrive_expect_tx(bar_t, P::kTwY + P::kTwX);
    if (!mod.starve) {
      bulk_g2s(tw_y, mod.stage_twiddle, P::kTwY, bar_t);
      bulk_g2s(tw_x, upd.stage_twiddle, P::kTwX, bar_t);
    }
  }
  __syncthreads();
  if (!__syncthreads_and(mbar_wait(bar_t, 0, mod.wait_tries) ? 1 : 0)) {
    if (tid == 0) {
      mbar_wait(bar_t, 0, mod.wait_tries);
      atomicAdd(mod.wait_failures, 1);
      atomicExch(abort, 1u);
    }
    return;
  }

  ColumnSmem cs;
  cs.box = sbase;
  cs.amp = sbase + P::CT::kRegion;
  cs.tw = tw_y;
  cs.bar = bar_c;
  cs.err_slot = err_slot;
  auto* w_tile = reinterpret_cast<float2*>(sbase);
  auto* x_tile = reinterpret_cast<float2*>(sbase + P::kRowW);
  auto* s_tile = sbase + P::kRowW + P::kRowX;
  unsigned parity_c = 0, parity_r = 0;

  for (;;) {
    if (tid == 0) {
      unsigned k = load_acquire(abort) ? total : atomicAdd(queue, 1u);
      *item_slot = k;
      int ok = 1;
      if (k < total) {
        const unsigned i = k / per_iteration;
        const unsigned rem = k - i * per_iteration;
        const unsigned modulus_items = static_cast<unsigned>(wl.starts) * wl.tiles_c;
        if (rem < modulus_items) {
          const unsigned s = rem / wl.tiles_c;
          ok = wait_count(done_r + s, i * wl.tiles_r, abort, mod.wait_tries);
        } else {
          const unsigned s = (rem - modulus_items) / wl.tiles_r;
          ok = wait_count(done_c + s, (i + 1) * wl.tiles_c, abort, mod.wait_tries);
        }
        if (!ok && !load_acquire(abort)) atomicAdd(mod.wait_failures, 1);
        if (!ok) atomicExch(abort, 1u);
        fence_proxy_async_global();  // the item's bulk loads follow the acquire
      }
      *flag_slot = ok;
    }
    __syncthreads();
    const unsigned k = *item_slot;
    if (k >= total || !*flag_slot) break;
    const unsigned i = k / per_iteration;
    const unsigned rem = k - i * per_iteration;
    const unsigned modulus_items = static_cast<unsigned>(wl.starts) * wl.tiles_c;
    bool ok;
    unsigned* done;
    if (rem < modulus_items) {
      ok = column_tile<LY, Mode::kMod, float, float2, kColumnLines, false>(
          &wmap, mod, static_cast<long long>(rem), cs, parity_c, row0 + static_cast<int>(i));
      parity_c ^= 1u;
      done = done_c + rem / wl.tiles_c;
    } else {
      const unsigned r = rem - modulus_items;
      ok = update_tile<LX, P::ROWS>(upd, static_cast<long long>(r), w_tile, x_tile, s_tile, tw_x,
                                    bar_w, bar_s, parity_r, ca, cb);
      parity_r ^= 1u;
      done = done_r + r / wl.tiles_r;
    }
    if (tid == 0) {
      if (!ok) {
        atomicExch(abort, 1u);
      } else {
        // the tile's stores complete and are published before its count
        bulk_wait_writes();
        fence_proxy_async_global();
        __threadfence();
        atomicAdd(done, 1u);
        if (atomicAdd(finished, 1u) == total - 1) {
          // the last item: the chunk's error rows are used up
          mod.ctrl->counters[mod.group] += wl.iterations;
        }
      }
    }
    __syncthreads();  // the shared memory is free for the next item
    if (!ok) break;
  }
}

template <int LY, int LX>
void launch_shape(const PassParams& mod, const PassParams& upd, int starts, int iterations,
                  unsigned* work, cudaStream_t stream) {
  using P = Persist<LY, LX>;
  static_assert(P::ROWS >= 1, "rows per update tile");
  const CUtensorMap map = column_wave_map(mod);
  WorkList wl{starts, iterations, LX / kColumnLines, LY / P::ROWS, work};
  int device = 0, sms = 0, per_sm = 0;
  QPB_CHECK(cudaGetDevice(&device));
  QPB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  QPB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_kernel<LY, LX>,
                                                          P::NT, P::kBytes));
  const long long items = static_cast<long long>(starts) * (wl.tiles_c + wl.tiles_r) * iterations;
  const int grid = static_cast<int>(std::min<long long>(static_cast<long long>(sms) * std::max(per_sm, 1),
                                                        items));
  cudaLaunchConfig_t config{};
  config.gridDim = dim3(static_cast<unsigned>(grid));
  config.blockDim = dim3(P::NT);
  config.dynamicSmemBytes = P::kBytes;
  config.stream = stream;
  // every CTA resident at once (the waits end without it; see above)
  cudaLaunchAttribute attr{};
  attr.id = cudaLaunchAttributeCooperative;
  attr.val.cooperative = 1;
  config.attrs = &attr;
  config.numAttrs = 1;
  QPB_CHECK(cudaLaunchKernelEx(&config, persistent_kernel<LY, LX>, map, mod, upd, wl));
  count_launches(1);
}

template <int LY, int LX>
void allow_shape() {
  constexpr int bytes = Persist<LY, LX>::kBytes;
  if constexpr (bytes > 48 * 1024) {
    QPB_CHECK(cudaFuncSetAttribute(persistent_kernel<LY, LX>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  }
}

template <int LY>
void launch_y(int lx, const PassParams& mod, const PassParams& upd, int starts, int iterations,
              unsigned* work, cudaStream_t stream) {
  switch (lx) {
    case 64: return launch_shape<LY, 64>(mod, upd, starts, iterations, work, stream);
    case 128: return launch_shape<LY, 128>(mod, upd, starts, iterations, work, stream);
    case 256: return launch_shape<LY, 256>(mod, upd, starts, iterations, work, stream);
    default: throw std::logic_error("persistent schedule: unsupported row length");
  }
}

template <int LY>
int grid_y(int lx) {
  auto grid = [](auto kernel, int nt, int bytes) {
    int device = 0, sms = 0, per_sm = 0;
    QPB_CHECK(cudaGetDevice(&device));
    QPB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    QPB_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nt, bytes));
    return sms * per_sm;
  };
  switch (lx) {
    case 64: return grid(persistent_kernel<LY, 64>, Persist<LY, 64>::NT, Persist<LY, 64>::kBytes);
    case 128: return grid(persistent_kernel<LY, 128>, Persist<LY, 128>::NT, Persist<LY, 128>::kBytes);
    case 256: return grid(persistent_kernel<LY, 256>, Persist<LY, 256>::NT, Persist<LY, 256>::kBytes);
    default: return 0;
  }
}

}  // namespace

bool persistent_supports(int ndim, int d1, int d2) {
  auto side = [](int n) { return n == 64 || n == 128 || n == 256; };
  return ndim == 2 && side(d1) && side(d2) && column_passes_enabled();
}

void launch_persistent(const PassParams& mod, const PassParams& upd, int starts, int iterations,
                       unsigned* work, cudaStream_t stream) {
  if (iterations < 1) return;
  if (mod.amp_tiled != kAmpTiledLines || mod.wave_half || upd.wave_half || upd.iter_half) {
    throw std::logic_error("persistent schedule: needs the line-major amplitude and complex64");
  }
  switch (mod.L) {
    case 64: return launch_y<64>(upd.L, mod, upd, starts, iterations, work, stream);
    case 128: return launch_y<128>(upd.L, mod, upd, starts, iterations, work, stream);
    case 256: return launch_y<256>(upd.L, mod, upd, starts, iterations, work, stream);
    default: throw std::logic_error("persistent schedule: unsupported column length");
  }
}

int persistent_grid(int d1, int d2) {
  switch (d1) {
    case 64: return grid_y<64>(d2);
    case 128: return grid_y<128>(d2);
    case 256: return grid_y<256>(d2);
    default: return 0;
  }
}

void configure_persistent() {
  static std::mutex mutex;
  static std::set<int> done;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  if (!done.insert(device).second) return;
  allow_shape<64, 64>();
  allow_shape<64, 128>();
  allow_shape<64, 256>();
  allow_shape<128, 64>();
  allow_shape<128, 128>();
  allow_shape<128, 256>();
  allow_shape<256, 64>();
  allow_shape<256, 128>();
  allow_shape<256, 256>();
}

}  // namespace qpb
