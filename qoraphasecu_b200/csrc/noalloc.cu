// Modulus projection that allocates no device memory.
//
// Some callers cannot call cudaMalloc: applications that reserve their whole
// GPU memory budget up front (a detector's streaming pipeline, a service whose
// memory pool already owns most of HBM) and must not grow it later, and
// latency-sensitive host threads for which cudaMalloc's implicit device
// synchronisation is not acceptable. For them, this file keeps the scratch the
// projection needs (signed amplitude, twiddle tables, control block, error
// accumulators) in one file-scope __device__ array of fixed size, and the
// caller passes every input and output as device memory.
//
// Limits: at most kNoAllocMaxElements elements per array, at most
// kNoAllocMaxLine along any axis. The array is shared by every call on a
// device and keeps the last call's contents (the twiddle tables of the last
// shape are reused by a call of the same shape); calls that overlap on the
// GPU race on it.

#include <array>
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>

#include "../../include/qpb.h"
#include "bulk_copy.cuh"
#include "fft_plan.hpp"
#include "line_pass.cuh"
#include "reduce.cuh"
#include "stage_table.hpp"

namespace qpb {

namespace {

constexpr long long kNoAllocMaxElements = 65536;  // e.g. 256 x 256 or 40 x 40 x 40
constexpr int kNoAllocMaxLine = 4096;

// Byte layout of the scratch array.
constexpr std::size_t kCtrlOffset = 0;       // Ctrl
constexpr std::size_t kCounterOffset = 64;   // int
constexpr std::size_t kErrOffset = 128;      // double: Fourier-error numerator
constexpr std::size_t kEnergyOffset = 136;   // double: usable energy
constexpr std::size_t kFailOffset = 144;     // int: line-pass CTAs whose bounded wait gave up
constexpr std::size_t kTwiddleOffset = 256;  // 3 axes x kNoAllocMaxLine float2
constexpr std::size_t kAmpOffset = kTwiddleOffset + 3 * kNoAllocMaxLine * sizeof(float2);
constexpr std::size_t kScratchBytes = kAmpOffset + kNoAllocMaxElements * sizeof(float);
static_assert(sizeof(Ctrl) <= kCounterOffset, "control block overlaps the counter");
static_assert(kNoAllocMaxLine >= 2 * 1024, "an axis slot holds W_L^k and the stage-major table");

__device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Per device: the scratch array's device address, looked up once (in host
// code `g_noalloc_scratch` is only a stand-in for the symbol, never an
// address), and the line length whose twiddle tables each axis slot holds, so
// that a call of the shape before rebuilds none of them.
struct ScratchState {
  unsigned char* base = nullptr;
  std::array<int, 3> table_length{0, 0, 0};
};

std::mutex g_scratch_mutex;

ScratchState& scratch_state() {
  static std::map<int, ScratchState> states;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  ScratchState& state = states[device];
  if (!state.base) {
    void* ptr = nullptr;
    QPB_CHECK(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    configure_line_passes();
    state.base = static_cast<unsigned char*>(ptr);
  }
  return state;
}

void require_aligned(const void* ptr, std::uintptr_t bytes, const char* name) {
  if (reinterpret_cast<std::uintptr_t>(ptr) % bytes != 0) {
    throw InvalidArgument(std::string("qpb_modulus_project_noalloc: ") + name +
                          " must be " + std::to_string(bytes) + "-byte aligned");
  }
}

// Resets the control block and the accumulators a call starts from.
__global__ void reset_kernel(unsigned char* base) {
  auto* ctrl = reinterpret_cast<Ctrl*>(base + kCtrlOffset);
  auto* counter = reinterpret_cast<int*>(base + kCounterOffset);
  *counter = 0;
  *reinterpret_cast<int*>(base + kFailOffset) = 0;
  *reinterpret_cast<double*>(base + kErrOffset) = 0.0;
  *reinterpret_cast<double*>(base + kEnergyOffset) = 0.0;
  ctrl->errs = reinterpret_cast<double*>(base + kErrOffset);
  ctrl->capacity = 1;
  ctrl->a = 0.0f;
  ctrl->b = 0.0f;
  ctrl->counters = counter;
}

// W_L^k = exp(-2 pi i k / L) from double-precision sincospi, rounded once.
__global__ void twiddle_kernel(float2* tw, int length) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < length; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-2.0 * static_cast<double>(k) / static_cast<double>(length), &s, &c);
    tw[k] = {static_cast<float>(c), static_cast<float>(s)};
  }
}

// The stage-major table of the register-resident passes (stage_table.hpp),
// copied entry by entry from the W_L^k table `tw` (stream order makes it ready).
__global__ void stage_twiddle_kernel(const float2* tw, float2* out, int length, StageGeometry g) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.count; i += gridDim.x * blockDim.x) {
    out[i] = tw[stage_twiddle_exponent(g, length, i)];
  }
}

// Signed amplitude (-1 on masked pixels) and the usable energy sum(A^2).
__global__ void signed_amplitude_kernel(const float* amp, const std::uint8_t* mask, float* out,
                                        long long n, double* energy) {
  double e = 0.0;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const bool masked = mask && mask[i];
    const float a = amp[i];
    out[i] = masked ? -1.0f : a;
    if (!masked) e += static_cast<double>(a) * a;
  }
  e = block_sum_double(e);
  if (threadIdx.x == 0) atomicAdd(energy, e);
}

// The Fourier error, or NaN when a line pass gave up a bounded wait (its CTAs
// wrote nothing, so `out` is not the projection).
__global__ void finalize_kernel(const double* num, const double* energy, const int* failures,
                                float* error_out) {
  *error_out = *failures ? __int_as_float(0x7fc00000)
                         : static_cast<float>(sqrt(*num / (*energy + static_cast<double>(kEps))));
}

void check_launch() {
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

}  // namespace

}  // namespace qpb

extern "C" qpb_status qpb_modulus_project_noalloc(int ndim, const int64_t* shape,
                                                  const float* amplitude, const uint8_t* mask,
                                                  const float* x, float* out, float* error_out,
                                                  void* stream) {
  using namespace qpb;
  try {
    clear_last_error();
    if (!shape || !amplitude || !x || !out || !error_out) {
      throw InvalidArgument("NULL argument");
    }
    // x and out are moved by bulk copies, which start on 16-byte boundaries.
    require_aligned(x, 16, "x");
    require_aligned(out, 16, "out");
    require_aligned(amplitude, alignof(float), "amplitude");
    require_aligned(error_out, alignof(float), "error_out");
    if (ndim != 2 && ndim != 3) {
      throw InvalidArgument("shape must be 2D or 3D, got ndim=" + std::to_string(ndim));
    }
    int dims[3] = {1, 1, 1};
    long long n = 1;
    for (int a = 0; a < ndim; ++a) {
      if (shape[a] < 1) throw InvalidArgument("shape has a zero-length axis");
      if (shape[a] > kNoAllocMaxLine) {
        throw InvalidArgument("qpb_modulus_project_noalloc: axis length " +
                              std::to_string(shape[a]) + " exceeds its maximum of " +
                              std::to_string(kNoAllocMaxLine));
      }
      dims[3 - ndim + a] = static_cast<int>(shape[a]);
      n *= shape[a];
    }
    if (n > kNoAllocMaxElements) {
      throw InvalidArgument("qpb_modulus_project_noalloc: " + std::to_string(n) +
                            " elements exceed its maximum of " +
                            std::to_string(kNoAllocMaxElements));
    }
    const auto s = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchState& state = scratch_state();
    unsigned char* base = state.base;
    auto* ctrl = reinterpret_cast<Ctrl*>(base + kCtrlOffset);
    auto* twiddles = reinterpret_cast<float2*>(base + kTwiddleOffset);
    auto* signed_amp = reinterpret_cast<float*>(base + kAmpOffset);

    reset_kernel<<<1, 1, 0, s>>>(base);
    check_launch();
    const int first_axis = ndim == 2 ? 1 : 0;
    PassParams axis_params[3] = {};
    for (int a = first_axis; a < 3; ++a) {
      const int L = dims[a];
      const auto radices = factorize(L);
      float2* tw = twiddles + a * kNoAllocMaxLine;
      const StageGeometry g = stage_geometry(L);
      if (state.table_length[a] != L) {
        twiddle_kernel<<<(L + 255) / 256, 256, 0, s>>>(tw, L);
        check_launch();
        if (g.count > 0) {
          // after the L entries of W_L^k in the axis's slot (L + count <= 2 L)
          stage_twiddle_kernel<<<(g.count + 255) / 256, 256, 0, s>>>(tw, tw + L, L, g);
          check_launch();
        }
        state.table_length[a] = L;
      }
      PassParams& p = axis_params[a];
      p.w = reinterpret_cast<float2*>(out);
      p.x = const_cast<float2*>(reinterpret_cast<const float2*>(x));
      p.amp = signed_amp;
      p.ctrl = ctrl;
      p.twiddle = tw;
      p.stage_twiddle = g.count > 0 ? tw + L : tw;
      p.n = n;
      p.L = L;
      p.S = a == 2 ? 1 : a == 1 ? dims[2] : dims[1] * dims[2];
      p.lines_per_start = static_cast<int>(n / L);
      p.lines = p.lines_per_start;
      p.lpc = choose_lpc(L, p.S, p.lines_per_start);
      p.stages = static_cast<int>(radices.size());
      for (int k = 0; k < p.stages; ++k) p.radix[k] = radices[k];
      p.scale = 1.0f / std::sqrt(static_cast<float>(n));
      p.starts_total = 1;
      p.amp_storage = AmpStorage::kF32;
      p.wait_tries = kMaxWaitTries;
      p.wait_failures = reinterpret_cast<int*>(base + kFailOffset);
    }
    signed_amplitude_kernel<<<static_cast<int>((n + 255) / 256), 256, 0, s>>>(
        amplitude, mask, signed_amp, n, reinterpret_cast<double*>(base + kEnergyOffset));
    check_launch();
    // Forward transform into `out`, modulus with the error, inverse in place.
    launch_line_pass(Mode::kFwdFromX, axis_params[2], s);
    if (ndim == 3) launch_line_pass(Mode::kFwd, axis_params[1], s);
    launch_line_pass(Mode::kMod, axis_params[first_axis], s);
    if (ndim == 3) launch_line_pass(Mode::kInv, axis_params[1], s);
    launch_line_pass(Mode::kInv, axis_params[2], s);
    finalize_kernel<<<1, 1, 0, s>>>(reinterpret_cast<const double*>(base + kErrOffset),
                                    reinterpret_cast<const double*>(base + kEnergyOffset),
                                    reinterpret_cast<const int*>(base + kFailOffset), error_out);
    check_launch();
    return QPB_OK;
  } catch (const std::invalid_argument& e) {
    set_last_error(e.what());
    return QPB_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return QPB_RUNTIME_ERROR;
  }
}
