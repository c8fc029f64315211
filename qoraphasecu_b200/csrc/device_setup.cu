// Problem set-up from arrays already on the device (callers holding torch or
// other device tensors): make_problem (src/core/problem.cpp:40-70) with the
// autocorrelation support (problem.cpp:72-88) computed on the device, and the
// per-problem preprocessing a solver needs (FFT-order roll, signed amplitude
// in its storage type and CTA tiling, usable energy), so no array crosses to
// the host.

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "device_setup.cuh"
#include "solver.hpp"

namespace qpb {

namespace {

constexpr int kThreads = 256;

int blocks_for(long long work) {
  return static_cast<int>(std::min<long long>(std::max<long long>((work + kThreads - 1) / kThreads, 1),
                                              148LL * 8));
}

#define QPB_LOOP(i, n)                                                              \
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; \
       i < (n); i += static_cast<long long>(gridDim.x) * blockDim.x)

// amplitude = sqrt(max(I, 0)); mask and support as 0/1; flags[0] counts
// non-finite intensities, flags[1] masked pixels.
__global__ void prepare_kernel(const float* intensity, const std::uint8_t* mask,
                               const std::uint8_t* support, long long n, float* amp,
                               std::uint8_t* mask_out, std::uint8_t* support_out,
                               unsigned long long* flags) {
  unsigned long long bad = 0, masked = 0;
  QPB_LOOP(i, n) {
    const float v = intensity[i];
    if (!isfinite(v)) ++bad;
    amp[i] = sqrtf(fmaxf(v, 0.0f));
    const std::uint8_t m = mask ? (mask[i] != 0) : 0;
    masked += m;
    mask_out[i] = m;
    if (support) support_out[i] = support[i] != 0;
  }
  if (bad) atomicAdd(flags, bad);
  if (masked) atomicAdd(flags + 1, masked);
}

__global__ void to_complex_kernel(const float* in, float2* out, long long n) {
  QPB_LOOP(i, n) out[i] = {in[i], 0.0f};
}

// |s w| (FFT order) and its maximum; |.| >= 0, so float bits order like values.
// Rounded step by step without contraction, exactly as the host computes it.
__global__ void magnitude_kernel(const float2* w, float* mag, long long n, float s,
                                 unsigned* max_bits) {
  float best = 0.0f;
  QPB_LOOP(i, n) {
    const float2 v = w[i];
    const float re = __fmul_rn(v.x, s), im = __fmul_rn(v.y, s);
    const float m = sqrtf(__fadd_rn(__fmul_rn(re, re), __fmul_rn(im, im)));
    mag[i] = m;
    best = fmaxf(best, m);
  }
  for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0) atomicMax(max_bits, __float_as_uint(best));
}

__global__ void threshold_kernel(const float* mag, long long n, const unsigned* max_bits,
                                 float threshold, std::uint8_t* out) {
  const float level = __fmul_rn(threshold, __uint_as_float(*max_bits));
  QPB_LOOP(i, n) out[i] = mag[i] > level;
}

// Element e (FFT order) of one problem goes to index `tiled(e)` of the
// signed-amplitude array: the modulus pass's CTA order for columns, element j
// of line c of CTA tile t at (t * L + j) * lines + c (element-major, the
// register-resident pass) or at (t * lines + c) * L + (j + r_c) mod L
// (line-major, the TMA column pass, r_c = amp_line_rotation(L, c)); FFT order
// otherwise.
__device__ __forceinline__ long long tiled_index(long long e, int L, int S, int lines,
                                                 bool line_major) {
  if (lines <= 0 || S == 1) return e;
  const long long slab = static_cast<long long>(L) * S;
  const long long outer = e / slab;
  const long long rem = e - outer * slab;
  const long long j = rem / S;
  const long long col = rem - j * S;
  const long long tile = outer * (S / lines) + col / lines;
  if (line_major) {
    const int line = static_cast<int>(col % lines);
    return (tile * lines + line) * L + ((j + amp_line_rotation(L, line)) & (L - 1));
  }
  return (tile * L + j) * lines + col % lines;
}

template <class T>
__device__ __forceinline__ T from_float(float v);
template <>
__device__ __forceinline__ float from_float<float>(float v) { return v; }
template <>
__device__ __forceinline__ __half from_float<__half>(float v) { return __float2half_rn(v); }
template <>
__device__ __forceinline__ __nv_bfloat16 from_float<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}

template <class T>
__global__ void signed_kernel(const float* amp, const std::uint8_t* mask, long long n, int L, int S,
                              int lines, bool line_major, T* out) {
  QPB_LOOP(e, n) {
    out[tiled_index(e, L, S, lines, line_major)] = from_float<T>(mask[e] ? -1.0f : amp[e]);
  }
}

__global__ void nonzero_kernel(std::uint8_t* v, long long n) {
  QPB_LOOP(i, n) v[i] = v[i] != 0;
}

// Usable energy, one block of kEnergyThreads: every element's share is added
// in the same order on every call.
constexpr int kEnergyThreads = 1024;

__global__ void __launch_bounds__(kEnergyThreads)
    energy_kernel(const float* amp, const std::uint8_t* mask, long long n, double* out) {
  __shared__ double partial[kEnergyThreads / 32];
  double e = 0.0;
  for (long long i = threadIdx.x; i < n; i += kEnergyThreads) {
    if (!mask[i]) e += static_cast<double>(amp[i]) * amp[i];
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kEnergyThreads / 32; ++w) t += partial[w];
    *out = t;
  }
}

// The amplitude's peak (one block; max of non-negative floats by their bits),
// then amp /= peak, for fp16 storage of the wave: with the peak amplitude at 1
// the stored transforms stay within fp16 range (the reference's
// src/cuda/cuda_solver.cu:74-86). A zero amplitude keeps scale 1.
__global__ void __launch_bounds__(kEnergyThreads)
    peak_kernel(const float* amp, long long n, float* peak) {
  __shared__ float partial[kEnergyThreads / 32];
  float m = 0.0f;
  for (long long i = threadIdx.x; i < n; i += kEnergyThreads) m = fmaxf(m, amp[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.0f;
    for (int w = 0; w < kEnergyThreads / 32; ++w) t = fmaxf(t, partial[w]);
    *peak = t > 0.0f ? t : 1.0f;
  }
}

__global__ void normalise_kernel(float* amp, long long n, const float* peak) {
  const float p = *peak;
  QPB_LOOP(i, n) amp[i] = amp[i] / p;
}

constexpr std::size_t align256(std::size_t bytes) { return (bytes + 255) / 256 * 256; }

// Device memory for problem set-up, one arena per device, grown on demand and
// kept for the process; set-up calls on one device take turns on it.
struct SetupArena {
  std::mutex mutex;
  std::unique_ptr<Stream> stream;
  DeviceBuffer<unsigned char> bytes;
  unsigned char* reserve(std::size_t count) {
    if (bytes.size() < count) {
      bytes = DeviceBuffer<unsigned char>();
      bytes = DeviceBuffer<unsigned char>(count);
    }
    return bytes.get();
  }
};

SetupArena& setup_arena() {
  static std::mutex mutex;
  static auto* arenas = new std::map<int, std::unique_ptr<SetupArena>>();  // never freed
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  auto& slot = (*arenas)[device];
  if (!slot) {
    slot = std::make_unique<SetupArena>();
    slot->stream = std::make_unique<Stream>();
  }
  return *slot;
}

std::size_t support_scratch_bytes(long long n) {
  const auto count = static_cast<std::size_t>(n);
  return 256 + 2 * align256(count * sizeof(float)) + align256(count * sizeof(float2));
}

// The autocorrelation support of a centre-origin device intensity into `out`
// (device): |IFFT(I)| in FFT order, centre-origin again, > threshold * max.
// `scratch`: support_scratch_bytes(n) device bytes.
void support_device(const float* intensity, Dims3 d, int ndim, float threshold, std::uint8_t* out,
                    unsigned char* scratch, cudaStream_t stream) {
  const long long n = d.n();
  const std::size_t plane = align256(static_cast<std::size_t>(n) * sizeof(float));
  auto* max_bits = reinterpret_cast<unsigned*>(scratch);
  auto* ordered = reinterpret_cast<float*>(scratch + 256);
  auto* mag = reinterpret_cast<float*>(scratch + 256 + plane);
  auto* w = reinterpret_cast<float2*>(scratch + 256 + 2 * plane);
  PassRunner runner(d, ndim, operator_plans());
  QPB_CHECK(cudaMemsetAsync(max_bits, 0, sizeof(unsigned), stream));
  roll<float>(intensity, ordered, d, 1, true, stream);
  to_complex_kernel<<<blocks_for(n), kThreads, 0, stream>>>(ordered, w, n);
  QPB_CHECK(cudaGetLastError());
  for (int axis3 = runner.outer(); axis3 < 3; ++axis3) {
    PassParams p = runner.params(Mode::kInv, axis3, 1);
    p.w = w;
    p.x = w;
    runner.launch(Mode::kInv, axis3, p, stream);
  }
  magnitude_kernel<<<blocks_for(n), kThreads, 0, stream>>>(
      w, ordered, n, 1.0f / std::sqrt(static_cast<float>(n)), max_bits);
  QPB_CHECK(cudaGetLastError());
  roll<float>(ordered, mag, d, 1, false, stream);
  threshold_kernel<<<blocks_for(n), kThreads, 0, stream>>>(mag, n, max_bits, threshold, out);
  QPB_CHECK(cudaGetLastError());
  count_launches(3);
}

}  // namespace

void make_problem_device(const float* intensity, int ndim, const long long* shape,
                         const std::uint8_t* support, const std::uint8_t* mask,
                         float support_threshold, float* amplitude_out, std::uint8_t* mask_out,
                         std::uint8_t* support_out, cudaStream_t stream) {
  ProblemView v;
  v.ndim = ndim;
  for (int a = 0; a < ndim && a < 3; ++a) v.shape[a] = shape[a];
  const Dims3 d = dims_of(v);
  const long long n = d.n();
  SetupArena& arena = setup_arena();
  std::lock_guard<std::mutex> lock(arena.mutex);
  unsigned char* scratch = arena.reserve(256 + (support ? 0 : support_scratch_bytes(n)));
  auto* flags = reinterpret_cast<unsigned long long*>(scratch);
  QPB_CHECK(cudaMemsetAsync(flags, 0, 2 * sizeof(unsigned long long), stream));
  prepare_kernel<<<blocks_for(n), kThreads, 0, stream>>>(intensity, mask, support, n, amplitude_out,
                                                          mask_out, support_out, flags);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
  if (!support) support_device(intensity, d, ndim, support_threshold, support_out, scratch + 256, stream);
  unsigned long long host_flags[2];
  QPB_CHECK(cudaMemcpyAsync(host_flags, flags, sizeof(host_flags), cudaMemcpyDeviceToHost, stream));
  QPB_CHECK(cudaStreamSynchronize(stream));
  check_waits(operator_plans(), stream);
  if (host_flags[0]) throw InvalidArgument("intensity contains NaN or Inf");
  if (mask && host_flags[1] == static_cast<unsigned long long>(n)) {
    throw InvalidArgument("mask marks every pixel as bad; nothing left to fit");
  }
}

void autocorrelation_support_host(const float* intensity, int ndim, const long long* shape,
                                  float threshold, std::uint8_t* out) {
  ProblemView v;
  v.ndim = ndim;
  if (ndim != 2 && ndim != 3) {
    throw InvalidArgument("shape must be 2D or 3D, got ndim=" + std::to_string(ndim));
  }
  for (int a = 0; a < ndim; ++a) v.shape[a] = shape[a];
  const Dims3 d = dims_of(v);
  const auto n = static_cast<std::size_t>(d.n());
  SetupArena& arena = setup_arena();
  std::lock_guard<std::mutex> lock(arena.mutex);
  const std::size_t in_bytes = align256(n * sizeof(float));
  unsigned char* scratch = arena.reserve(in_bytes + align256(n) + support_scratch_bytes(d.n()));
  auto* dev_in = reinterpret_cast<float*>(scratch);
  std::uint8_t* dev_out = scratch + in_bytes;
  const cudaStream_t s = *arena.stream;
  QPB_CHECK(cudaMemcpyAsync(dev_in, intensity, n * sizeof(float), cudaMemcpyHostToDevice, s));
  support_device(dev_in, d, ndim, threshold, dev_out, scratch + in_bytes + align256(n), s);
  QPB_CHECK(cudaMemcpyAsync(out, dev_out, n, cudaMemcpyDeviceToHost, s));
  QPB_CHECK(cudaStreamSynchronize(s));
  check_waits(operator_plans(), s);
}

std::size_t prepare_scratch_bytes(long long n) { return align256(static_cast<std::size_t>(n)); }

void prepare_problem_device(const ProblemView& q, Dims3 d, AmpStorage storage, int L, int S,
                            int lines, bool line_major, float* amp_fft, void* signed_out,
                            std::uint8_t* support_fft, void* scratch, double* energy,
                            float* peak, cudaStream_t stream) {
  const long long n = d.n();
  std::uint8_t* mask_fft = static_cast<std::uint8_t*>(scratch);
  roll<float>(q.amplitude, amp_fft, d, 1, true, stream);
  if (peak) {
    peak_kernel<<<1, kEnergyThreads, 0, stream>>>(amp_fft, n, peak);
    QPB_CHECK(cudaGetLastError());
    normalise_kernel<<<blocks_for(n), kThreads, 0, stream>>>(amp_fft, n, peak);
    QPB_CHECK(cudaGetLastError());
    count_launches(2);
  }
  if (q.mask) {
    roll<std::uint8_t>(q.mask, mask_fft, d, 1, true, stream);
  } else {
    QPB_CHECK(cudaMemsetAsync(mask_fft, 0, static_cast<std::size_t>(n), stream));
  }
  roll<std::uint8_t>(q.support, support_fft, d, 1, true, stream);
  nonzero_kernel<<<blocks_for(n), kThreads, 0, stream>>>(support_fft, n);
  QPB_CHECK(cudaGetLastError());
  switch (storage) {
    case AmpStorage::kF32:
      signed_kernel<float><<<blocks_for(n), kThreads, 0, stream>>>(
          amp_fft, mask_fft, n, L, S, lines, line_major, static_cast<float*>(signed_out));
      break;
    case AmpStorage::kF16:
      signed_kernel<__half><<<blocks_for(n), kThreads, 0, stream>>>(
          amp_fft, mask_fft, n, L, S, lines, line_major, static_cast<__half*>(signed_out));
      break;
    case AmpStorage::kBF16:
      signed_kernel<__nv_bfloat16><<<blocks_for(n), kThreads, 0, stream>>>(
          amp_fft, mask_fft, n, L, S, lines, line_major, static_cast<__nv_bfloat16*>(signed_out));
      break;
  }
  QPB_CHECK(cudaGetLastError());
  energy_kernel<<<1, kEnergyThreads, 0, stream>>>(amp_fft, mask_fft, n, energy);
  QPB_CHECK(cudaGetLastError());
  count_launches(3);
}

}  // namespace qpb
