// Column line passes (stride S > 1) whose tiles move by TMA.
//
// A CTA owns LINES adjacent columns of one outer slab: a [L][LINES] complex64
// box of the wave. One tensor-map copy (cp.async.bulk.tensor, 3D map over the
// launch's wave: {S, L, outer slabs}) brings the whole box into shared memory,
// swizzled so that the row-order reads below are free of bank conflicts; a
// modulus pass's amplitude tile (stored by the problem set-up in this pass's
// CTA order, line-major) and the transform's stage-major twiddle table arrive
// by bulk copies on the same mbarrier.
//
// Inside the CTA the lines are held row-style: the T threads of a line sit in
// one warp (thread t of line l owns elements t + T m), so every Stockham
// exchange of the register-resident transform (line_fft.cuh) needs a warp
// barrier only, and the Fourier-error sum is a warp reduction with one FP64
// atomic per warp. The result goes back through the same swizzled box and
// leaves by one tensor-map store. Block barriers: one after the box is read
// into registers (the box becomes the exchange rows) and two around the
// output box.
//
// Every wait is bounded (PassParams::wait_tries); a CTA that gives up waits
// once more for its copies in flight, counts itself in p.wait_failures and
// writes nothing.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>

#include "bulk_copy.cuh"
#include "column_pass.cuh"
#include "line_fft.cuh"
#include "projection.cuh"
#include "reduce.cuh"
#include "storage.cuh"

namespace qpb {

namespace {

// Lines per CTA of every column pass: 8 (the default), or 16 when the
// environment sets QPB_COLUMN_LINES=16 (both are built; used to compare them).
int column_lines() {
  static const int lines = [] {
    const char* v = std::getenv("QPB_COLUMN_LINES");
    return v && std::atoi(v) == 16 ? 16 : 8;
  }();
  return lines;
}

// CTA shape: LINES_ columns of L points, T threads a line, the wave stored as
// WT (float2 or __half2). A box row is LINES_ elements: 64 or 128 bytes of
// complex64, 32 or 64 of fp16 pairs, swizzled with the pattern of that width.
// The register budget is sized for MIN_CTAS resident CTAs per SM
// (registers <= 64K / (NT * MIN_CTAS)): at 8 lines all CTAs of a 32-start
// 256 x 256 launch fit in one wave.
template <int L, class WT, int LINES_>
struct ColumnTiling {
  using G = Geometry<L>;
  static constexpr int LINES = LINES_;
  static constexpr int NT = G::T * LINES;
  static constexpr int MIN_CTAS = NT <= 64 ? 12 : (NT <= 128 ? 7 : 3);
  static constexpr int ROW_BYTES = LINES * static_cast<int>(sizeof(WT));  // one box row
  static constexpr int kBox = L * ROW_BYTES;
  static constexpr int kExchange = LINES * G::PITCH * 8;
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

template <int L, Mode M, class AmpT, class WT, int LINES_>
__global__ void __launch_bounds__(ColumnTiling<L, WT, LINES_>::NT,
                                  ColumnTiling<L, WT, LINES_>::MIN_CTAS)
    column_pass_kernel(const __grid_constant__ CUtensorMap wmap, const PassParams p) {
  using G = Geometry<L>;
  using Ti = ColumnTiling<L, WT, LINES_>;
  using St = ColumnStaging<L, M, AmpT, WT, LINES_>;
  constexpr int E = G::E;
  constexpr int T = G::T;
  constexpr int LINES = Ti::LINES;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sbase = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<std::uintptr_t>(smem_raw) + 1023) & ~static_cast<std::uintptr_t>(1023));
  unsigned char* box = sbase;
  auto* bar = reinterpret_cast<std::uint64_t*>(sbase + St::kBarrier);

  const int tid = threadIdx.x;
  const int l = tid / T;  // line within the CTA
  const int t = tid % T;  // thread within the line
  const long long line0 = static_cast<long long>(blockIdx.x) * LINES;
  const int outer = static_cast<int>(line0 / p.S);
  const int inner0 = static_cast<int>(line0 - static_cast<long long>(outer) * p.S);
  const int batch_start = static_cast<int>(line0 / p.lines_per_start);

  if (tid == 0) {
    mbar_init(bar, 1);
    mbar_arrive_expect_tx(bar, St::kAmpBytes + St::kTwBytes + Ti::kBox);
    if (!p.starve) {
      tma_load_3d(box, &wmap, inner0, 0, outer, bar);
      bulk_g2s(sbase + St::kTwOffset, p.stage_twiddle, St::kTwBytes, bar);
      if constexpr (St::kAmp) {
        const long long line_in_start =
            line0 - static_cast<long long>(batch_start) * p.lines_per_start;
        const AmpT* src = static_cast<const AmpT*>(p.amp) + amp_offset(p, p.start0 + batch_start) +
                          line_in_start * L;
        bulk_g2s(sbase + St::kAmpOffset, src, St::kAmpBytes, bar);
      }
    }
  }
  // Control values while the copies are in flight: a modulus pass's error
  // row, kept in shared memory (next to the barrier) until the sum is ready.
  auto* err_slot = reinterpret_cast<double**>(sbase + St::kBarrier + 8);
  if constexpr (M == Mode::kMod) {
    if (tid == 0) {
      const Ctrl* c = p.ctrl;
      const int r = c->counters[p.group];
      *err_slot = r < c->capacity
                      ? c->errs + static_cast<long long>(r) * p.starts_total + p.start0 + batch_start
                      : nullptr;
    }
  }
  const float2* tw = reinterpret_cast<const float2*>(sbase + St::kTwOffset);
  __syncthreads();  // the barrier is initialised before anyone polls it

  if (!__syncthreads_and(mbar_wait(bar, 0, p.wait_tries) ? 1 : 0)) {
    if (tid == 0) {
      mbar_wait(bar, 0, p.wait_tries);  // copies still in flight land first
      atomicAdd(p.wait_failures, 1);
    }
    return;
  }

  float2 v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int j = t + T * m;
    v[m] = load_c(*reinterpret_cast<const WT*>(
        box + swizzled<Ti::ROW_BYTES>(j * Ti::ROW_BYTES + l * static_cast<int>(sizeof(WT)))));
  }
  __syncthreads();  // the box becomes the lines' exchange rows
  float2* row = reinterpret_cast<float2*>(box) + l * G::PITCH;

  if constexpr (M == Mode::kMod) {
    transform<L, false, true, true, true>(v, t, tw, row);
    const AmpT* amp_tile = reinterpret_cast<const AmpT*>(sbase + St::kAmpOffset) + l * L;
    const float s = p.scale;
    float acc = 0.0f;
#pragma unroll
    for (int m = 0; m < E; ++m) {
      // an fp16 wave defers the inverse's 1/sqrt(n) to the update pass
      v[m] = pointwise_projection<Mode::kMod>(v[m], to_float(amp_tile[t + T * m]), s, acc,
                                              kHalfStorage<WT> ? 1.0f : s);
    }
    // every line of the CTA belongs to one start: one atomic per warp
    const double total = warp_sum_double(static_cast<double>(acc));
    if ((tid & 31) == 0) {
      double* slot = *err_slot;
      if (slot) atomicAdd(slot, total);
    }
    transform<L, true, true, true, true>(v, t, tw, row);
  } else {
    transform<L, M == Mode::kInv, true, true, true>(v, t, tw, row);
  }

  __syncthreads();  // every line is done with the exchange rows
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int j = t + T * m;
    *reinterpret_cast<WT*>(box + swizzled<Ti::ROW_BYTES>(
        j * Ti::ROW_BYTES + l * static_cast<int>(sizeof(WT)))) = store_c<WT>(v[m]);
  }
  fence_proxy_async();
  __syncthreads();
  if (tid == 0) {
    tma_store_3d(&wmap, inner0, 0, outer, box);
    bulk_commit();
    bulk_wait_reads();
  }
}

// ------------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult query{};
    QPB_CHECK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &query));
    if (query != cudaDriverEntryPointSuccess || !ptr) {
      throw std::runtime_error("cuTensorMapEncodeTiled is not available from the driver");
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  }();
  return fn;
}

// The launch's wave as a 3D tensor {S, L, outer slabs} of 8-byte (complex64)
// or 4-byte (fp16 pair) elements and its [1][L][LINES] box.
template <int L, class WT, int LINES>
CUtensorMap wave_map(const PassParams& p) {
  using Ti = ColumnTiling<L, WT, LINES>;
  constexpr cuuint64_t kElem = sizeof(WT);
  CUtensorMap map{};
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(p.S), static_cast<cuuint64_t>(L),
                              static_cast<cuuint64_t>(p.lines / p.S)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(p.S) * kElem,
                                 static_cast<cuuint64_t>(p.S) * L * kElem};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(Ti::LINES), static_cast<cuuint32_t>(L), 1};
  const cuuint32_t estrides[3] = {1, 1, 1};
  const CUresult r = encode_fn()(
      &map, kElem == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, p.w,
      dims, strides, box, estrides, CU_TENSOR_MAP_INTERLEAVE_NONE,
      swizzle_mode<Ti::ROW_BYTES>(),
      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    throw std::runtime_error("cuTensorMapEncodeTiled failed for a column pass (code " +
                             std::to_string(static_cast<int>(r)) + ")");
  }
  return map;
}

template <int L, Mode M, class AmpT, class WT, int LINES>
void launch_lines(const PassParams& p, cudaStream_t stream) {
  using Ti = ColumnTiling<L, WT, LINES>;
  const CUtensorMap map = wave_map<L, WT, LINES>(p);
  const dim3 grid(static_cast<unsigned>(p.lines / Ti::LINES));
  column_pass_kernel<L, M, AmpT, WT, LINES>
      <<<grid, Ti::NT, ColumnStaging<L, M, AmpT, WT, LINES>::kBytes, stream>>>(map, p);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

template <int L, Mode M, class AmpT, class WT>
void launch_one(const PassParams& p, cudaStream_t stream) {
  if (column_lines() == 16) return launch_lines<L, M, AmpT, WT, 16>(p, stream);
  launch_lines<L, M, AmpT, WT, 8>(p, stream);
}

template <int L, Mode M>
void launch_storage(const PassParams& p, cudaStream_t stream) {
  if (p.wave_half) {
    if (p.amp_storage != AmpStorage::kF32) {
      throw std::logic_error("column pass: an fp16 wave runs with an FP32 amplitude");
    }
    return launch_one<L, M, float, __half2>(p, stream);
  }
  if constexpr (M == Mode::kMod) {
    switch (p.amp_storage) {
      case AmpStorage::kF32:
        return launch_one<L, M, float, float2>(p, stream);
      case AmpStorage::kF16:
        return launch_one<L, M, __half, float2>(p, stream);
      case AmpStorage::kBF16:
        return launch_one<L, M, __nv_bfloat16, float2>(p, stream);
    }
  } else {
    launch_one<L, M, float, float2>(p, stream);
  }
}

template <int L>
void launch_length(Mode mode, const PassParams& p, cudaStream_t stream) {
  switch (mode) {
    case Mode::kMod:
      return launch_storage<L, Mode::kMod>(p, stream);
    case Mode::kFwd:
      return launch_storage<L, Mode::kFwd>(p, stream);
    case Mode::kInv:
      return launch_storage<L, Mode::kInv>(p, stream);
    default:
      throw std::logic_error("column pass: unsupported mode");
  }
}

template <int L, Mode M, class AmpT, class WT, int LINES>
void allow_lines() {
  constexpr int bytes = ColumnStaging<L, M, AmpT, WT, LINES>::kBytes;
  if constexpr (bytes > 48 * 1024) {
    QPB_CHECK(cudaFuncSetAttribute(column_pass_kernel<L, M, AmpT, WT, LINES>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  }
}

template <int L, Mode M, class AmpT, class WT = float2>
void allow_one() {
  allow_lines<L, M, AmpT, WT, 8>();
  allow_lines<L, M, AmpT, WT, 16>();
}

template <int L>
void allow_length() {
  allow_one<L, Mode::kMod, float>();
  allow_one<L, Mode::kMod, __half>();
  allow_one<L, Mode::kMod, __nv_bfloat16>();
  allow_one<L, Mode::kFwd, float>();
  allow_one<L, Mode::kInv, float>();
  allow_one<L, Mode::kMod, float, __half2>();
  allow_one<L, Mode::kFwd, float, __half2>();
  allow_one<L, Mode::kInv, float, __half2>();
}

}  // namespace

bool column_passes_enabled() {
  static const bool enabled = [] {
    const char* v = std::getenv("QPB_COLUMN_PASSES");
    return !(v && *v == '0');
  }();
  return enabled;
}

int column_pass_lines(const PassParams& p, Mode mode) {
  if (!column_passes_enabled() || p.S <= 1) return 0;
  if (p.L != 64 && p.L != 128 && p.L != 256) return 0;
  if (mode != Mode::kMod && mode != Mode::kFwd && mode != Mode::kInv) return 0;
  if (mode == Mode::kMod && p.amp_tiled != kAmpTiledLines) return 0;
  const int lines = column_lines();
  if (p.S % lines != 0 || p.lines_per_start % lines != 0 || p.lines % lines != 0) return 0;
  if (p.lines % p.S != 0) return 0;
  if (reinterpret_cast<std::uintptr_t>(p.w) % 16 != 0) return 0;
  return lines;
}

void launch_column_pass(Mode mode, const PassParams& p, cudaStream_t stream) {
  switch (p.L) {
    case 64:
      return launch_length<64>(mode, p, stream);
    case 128:
      return launch_length<128>(mode, p, stream);
    case 256:
      return launch_length<256>(mode, p, stream);
    default:
      throw std::logic_error("column pass: unsupported length");
  }
}

void configure_column_passes() {
  static std::mutex mutex;
  static std::set<int> done;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  if (!done.insert(device).second) return;
  allow_length<64>();
  allow_length<128>();
  allow_length<256>();
}

}  // namespace qpb
