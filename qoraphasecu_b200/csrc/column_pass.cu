// Column line passes (stride S > 1) whose tiles move by TMA: one tile of
// column_tile.cuh per CTA (LINES adjacent columns as one [L][LINES] box of a
// 3D tensor map over the launch's wave, {S, L, outer slabs}; lines of 512
// points as two boxes of 256 rows); this file holds the kernel, the
// tensor-map encoding and the launch dispatch.
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
#include <map>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>

#include "column_pass.cuh"
#include "column_tile.cuh"
#include "dependent_launch.cuh"

namespace qpb {

namespace {

// Lines per CTA of every column pass (16 measured slower: 14.8 against 14.2 us
// for the 256^2 modulus pass of 32 starts).
constexpr int kLines = 8;

// Resident CTAs per SM of the wide variant of the 256-point modulus pass
// (complex64 wave): 72 registers a thread, no spills, against 93 at the
// default 5 per SM. A launch of 32 starts (1024 CTAs) then runs in one wave
// of 148 SMs: 10.75 against 11.37 us, and 128 starts 31.0 against 33.1 us.
// Launches that fit one wave at the default occupancy keep the default
// variant, which runs fewer instructions a tile: with start groups of 4 as 8
// concurrent graph branches the wide variant made an iteration of 32 starts
// 5% slower (17.65 against 16.83 us).
constexpr int kWideCtas = 7;

template <int L, Mode M, class WT>
constexpr bool kHasWide = L == 256 && M == Mode::kMod && std::is_same_v<WT, float2>;

// One tile per CTA; CTAS resident CTAs per SM bound the registers.
template <int L, Mode M, class AmpT, class WT, int LINES_, int CTAS>
__global__ void __launch_bounds__(ColumnTiling<L, WT, LINES_>::NT, CTAS)
    column_pass_kernel(const __grid_constant__ CUtensorMap wmap, const PassParams p) {
  using St = ColumnStaging<L, M, AmpT, WT, LINES_>;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sbase = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<std::uintptr_t>(smem_raw) + 1023) & ~static_cast<std::uintptr_t>(1023));
  ColumnSmem s;
  s.box = sbase;
  s.amp = sbase + St::kAmpOffset;
  s.tw = reinterpret_cast<const float2*>(sbase + St::kTwOffset);
  s.bar = reinterpret_cast<std::uint64_t*>(sbase + St::kBarrier);
  s.err_slot = reinterpret_cast<double**>(sbase + St::kBarrier + 8);
  if (threadIdx.x == 0) mbar_init(s.bar, 1);
  __syncthreads();  // the barrier is initialised before anyone polls it
  wait_for_prior_kernel();  // the wave and the control block come from it
  allow_next_kernel();
  if (column_tile<L, M, AmpT, WT, LINES_, true>(&wmap, p, blockIdx.x, s, 0, -1)) {
    if (threadIdx.x == 0) bulk_wait_reads();
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
// or 4-byte (fp16 pair) elements and its [1][kBoxRows][LINES] box (a tile of
// a line longer than 256 points takes several boxes).
template <int L, class WT, int LINES>
CUtensorMap wave_map(const PassParams& p) {
  using Ti = ColumnTiling<L, WT, LINES>;
  constexpr cuuint64_t kElem = sizeof(WT);
  CUtensorMap map{};
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(p.S), static_cast<cuuint64_t>(L),
                              static_cast<cuuint64_t>(p.lines / p.S)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(p.S) * kElem,
                                 static_cast<cuuint64_t>(p.S) * L * kElem};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(Ti::LINES),
                             static_cast<cuuint32_t>(Ti::kBoxRows), 1};
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

// Encoded tensor maps of this thread, by wave address and geometry: encoding
// validates the whole description on the host, which a direct launch (the
// plain variant, per-pass timing) would otherwise pay on every launch.
struct MapKey {
  const void* base;
  long long lines;
  int S, L, elem, lines_per_cta;
  bool operator<(const MapKey& o) const {
    return std::tie(base, lines, S, L, elem, lines_per_cta) <
           std::tie(o.base, o.lines, o.S, o.L, o.elem, o.lines_per_cta);
  }
};

template <int L, class WT, int LINES>
const CUtensorMap& cached_wave_map(const PassParams& p) {
  thread_local std::map<MapKey, CUtensorMap> cache;
  const MapKey key{p.w, p.lines, p.S, L, static_cast<int>(sizeof(WT)), LINES};
  auto it = cache.find(key);
  if (it == cache.end()) {
    if (cache.size() >= 256) cache.clear();  // buffers come and go; keep the cache small
    it = cache.emplace(key, wave_map<L, WT, LINES>(p)).first;
  }
  return it->second;
}

// Multiprocessors of the current device (cached per device).
int device_sms() {
  static std::mutex mutex;
  static std::map<int, int> sms;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  const std::lock_guard<std::mutex> lock(mutex);
  auto it = sms.find(device);
  if (it == sms.end()) {
    int n = 0;
    QPB_CHECK(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device));
    it = sms.emplace(device, n).first;
  }
  return it->second;
}

template <int L, Mode M, class AmpT, class WT, int LINES>
void launch_lines(const PassParams& p, cudaStream_t stream) {
  using Ti = ColumnTiling<L, WT, LINES>;
  constexpr int kBytes = ColumnStaging<L, M, AmpT, WT, LINES>::kBytes;
  const CUtensorMap& map = cached_wave_map<L, WT, LINES>(p);
  const long long ctas = p.lines / Ti::LINES;
  const dim3 grid(static_cast<unsigned>(ctas));
  if constexpr (kHasWide<L, M, WT>) {
    if (ctas > static_cast<long long>(Ti::MIN_CTAS) * device_sms()) {
      launch_dependent(column_pass_kernel<L, M, AmpT, WT, LINES, kWideCtas>, grid, dim3(Ti::NT),
                       kBytes, stream, map, p);
      count_launches(1);
      return;
    }
  }
  launch_dependent(column_pass_kernel<L, M, AmpT, WT, LINES, Ti::MIN_CTAS>, grid, dim3(Ti::NT),
                   kBytes, stream, map, p);
  count_launches(1);
}

template <int L, Mode M, class AmpT, class WT>
void launch_one(const PassParams& p, cudaStream_t stream) {
  launch_lines<L, M, AmpT, WT, kLines>(p, stream);
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
    QPB_CHECK(cudaFuncSetAttribute(
        column_pass_kernel<L, M, AmpT, WT, LINES, ColumnTiling<L, WT, LINES>::MIN_CTAS>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    if constexpr (kHasWide<L, M, WT>) {
      QPB_CHECK(cudaFuncSetAttribute(column_pass_kernel<L, M, AmpT, WT, LINES, kWideCtas>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    }
  }
}

template <int L, Mode M, class AmpT, class WT = float2>
void allow_one() {
  allow_lines<L, M, AmpT, WT, kLines>();
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

CUtensorMap column_wave_map(const PassParams& p) {
  switch (p.L) {
    case 64:
      return cached_wave_map<64, float2, kLines>(p);
    case 128:
      return cached_wave_map<128, float2, kLines>(p);
    case 256:
      return cached_wave_map<256, float2, kLines>(p);
    default:
      throw std::logic_error("column pass: unsupported length");
  }
}

bool column_passes_enabled() {
  static const bool enabled = [] {
    const char* v = std::getenv("QPB_COLUMN_PASSES");
    return !(v && *v == '0');
  }();
  return enabled;
}

int column_pass_lines(const PassParams& p, Mode mode) {
  if (!column_passes_enabled() || p.S <= 1) return 0;
  if (p.L != 64 && p.L != 128 && p.L != 256 && p.L != 512) return 0;
  if (mode != Mode::kMod && mode != Mode::kFwd && mode != Mode::kInv) return 0;
  if (mode == Mode::kMod && p.amp_tiled != kAmpTiledLines) return 0;
  constexpr int lines = kLines;
  if (p.S % lines != 0 || p.lines_per_start % lines != 0 || p.lines % lines != 0) return 0;
  if (p.lines % p.S != 0) return 0;
  if (reinterpret_cast<std::uintptr_t>(p.w) % 16 != 0) return 0;
  return lines;
}

bool column_pass_preferred(const PassParams& p, Mode mode) {
  return p.L >= 128 && column_pass_lines(p, mode) > 0;
}

void launch_column_pass(Mode mode, const PassParams& p, cudaStream_t stream) {
  switch (p.L) {
    case 64:
      return launch_length<64>(mode, p, stream);
    case 128:
      return launch_length<128>(mode, p, stream);
    case 256:
      return launch_length<256>(mode, p, stream);
    case 512:
      return launch_length<512>(mode, p, stream);
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
  allow_length<512>();
}

}  // namespace qpb
