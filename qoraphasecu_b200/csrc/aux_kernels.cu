#include <cuda_fp16.h>

#include <algorithm>

#include <stdexcept>

#include "aux_kernels.cuh"
#include "common.cuh"
#include "reduce.cuh"

namespace qpb {

namespace {

constexpr int kThreads = 256;

int blocks_for(long long work) {
  return static_cast<int>(std::min<long long>(std::max<long long>((work + kThreads - 1) / kThreads, 1),
                                              148LL * 16));
}

// A grid-stride loop over `work` items with the start in blockIdx.y.
#define QPB_FOR(i, work)                                                            \
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; \
       i < (work); i += static_cast<long long>(gridDim.x) * blockDim.x)

__global__ void random_wave_kernel(float2* w, const float* amp, long long amp_stride,
                                   int starts_per_problem, long long n, std::uint64_t seed,
                                   std::uint64_t first_start) {
  const float s = rsqrtf(static_cast<float>(n));
  const std::uint64_t global = first_start + blockIdx.y;
  // Each problem's starts are keyed 0, 1, ... as if it ran alone.
  const std::uint64_t start = global % static_cast<std::uint64_t>(starts_per_problem);
  amp += static_cast<long long>(global / static_cast<std::uint64_t>(starts_per_problem)) * amp_stride;
  w += blockIdx.y * n;
  QPB_FOR(i, n) {
    const float phase = kTwoPi * uniform(seed, start, static_cast<std::uint64_t>(i));
    const float a = amp[i] * s;
    float sn, cs;
    sincosf(phase, &sn, &cs);
    w[i] = {a * cs, a * sn};
  }
}

__global__ void support_project_kernel(float2* x, const std::uint8_t* support, long long n) {
  x += blockIdx.y * n;
  support += blockIdx.y * n;
  QPB_FOR(i, n) {
    if (!support[i]) x[i] = {0.0f, 0.0f};
  }
}

__global__ void threshold_kernel(const float2* blurred, const LevelAcc* acc, long long n,
                                 int method, float threshold, std::uint8_t* support) {
  const LevelAcc& a = acc[blockIdx.y];
  const float level = method == 1
                          ? __int_as_float(a.max_bits)
                          : static_cast<float>(sqrt(a.sum / fmax(static_cast<double>(a.count), 1.0)));
  const float cut = threshold * level;
  blurred += blockIdx.y * n;
  support += blockIdx.y * n;
  QPB_FOR(i, n) { support[i] = blurred[i].x > cut; }
}

// Centre-origin coordinate along a Dims3 axis of FFT-order flat index i.
__device__ __forceinline__ int centred_coord(long long i, Dims3 d, int axis3) {
  long long c;
  int len;
  if (axis3 == 2) {
    c = i % d.d2;
    len = d.d2;
  } else if (axis3 == 1) {
    c = (i / d.d2) % d.d1;
    len = d.d1;
  } else {
    c = i / (static_cast<long long>(d.d1) * d.d2);
    len = d.d0;
  }
  return static_cast<int>((c + len / 2) % len);
}

__global__ void detwin_moment_kernel(const std::uint8_t* support, Dims3 d, int axis3,
                                     unsigned long long* moments) {
  const long long n = d.n();
  support += blockIdx.y * n;
  unsigned long long moment = 0, weight = 0;
  QPB_FOR(i, n) {
    if (support[i]) {
      moment += static_cast<unsigned long long>(centred_coord(i, d, axis3));
      ++weight;
    }
  }
  const double m = block_sum_double(static_cast<double>(moment));
  __syncthreads();
  const double w = block_sum_double(static_cast<double>(weight));
  if (threadIdx.x == 0) {
    atomicAdd(&moments[2 * blockIdx.y], static_cast<unsigned long long>(m));
    atomicAdd(&moments[2 * blockIdx.y + 1], static_cast<unsigned long long>(w));
  }
}

__global__ void detwin_apply_kernel(std::uint8_t* support, Dims3 d, int axis3,
                                    const unsigned long long* moments) {
  const long long n = d.n();
  support += blockIdx.y * n;
  // half_support's FP64 centre of mass of exact integer sums.
  const double centre = static_cast<double>(moments[2 * blockIdx.y]) /
                        fmax(static_cast<double>(moments[2 * blockIdx.y + 1]), 1.0);
  QPB_FOR(i, n) {
    if (support[i] && !(static_cast<double>(centred_coord(i, d, axis3)) < centre)) support[i] = 0;
  }
}

template <class T>
__global__ void roll_kernel(const T* in, T* out, Dims3 d, int o0, int o1, int o2) {
  const long long n = d.n();
  in += blockIdx.y * n;
  out += blockIdx.y * n;
  QPB_FOR(i, n) {
    const int x = static_cast<int>(i % d.d2);
    const int y = static_cast<int>((i / d.d2) % d.d1);
    const int z = static_cast<int>(i / (static_cast<long long>(d.d1) * d.d2));
    const int sz = (z + o0) % d.d0;
    const int sy = (y + o1) % d.d1;
    const int sx = (x + o2) % d.d2;
    out[i] = in[(static_cast<long long>(sz) * d.d1 + sy) * d.d2 + sx];
  }
}

__global__ void set_coefficients_kernel(Ctrl* ctrl, float a, float b) {
  ctrl->a = a;
  ctrl->b = b;
}

__global__ void set_ctrl_kernel(Ctrl* ctrl, Ctrl value) { *ctrl = value; }

__global__ void scale_complex_kernel(float2* x, long long count, float scale) {
  QPB_FOR(i, count) { x[i] = cscale(x[i], scale); }
}

__global__ void to_half_kernel(const float2* in, __half2* out, long long count) {
  QPB_FOR(i, count) { out[i] = __float22half2_rn(in[i]); }
}

__global__ void from_half_kernel(const __half2* in, float2* out, long long count) {
  QPB_FOR(i, count) { out[i] = __half22float2(in[i]); }
}

dim3 grid(long long n, int batch) {
  return {static_cast<unsigned>(blocks_for(n)), static_cast<unsigned>(batch), 1};
}

}  // namespace

void random_wave(float2* w, const float* amplitude, long long amp_stride, int starts_per_problem,
                 long long n, int batch, std::uint64_t seed, std::uint64_t first_start,
                 cudaStream_t stream) {
  if (starts_per_problem < 1) throw std::logic_error("random_wave: starts_per_problem < 1");
  random_wave_kernel<<<grid(n, batch), kThreads, 0, stream>>>(w, amplitude, amp_stride,
                                                              starts_per_problem, n, seed,
                                                              first_start);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

void support_project(float2* x, const std::uint8_t* support, long long n, int batch,
                     cudaStream_t stream) {
  support_project_kernel<<<grid(n, batch), kThreads, 0, stream>>>(x, support, n);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

void shrinkwrap_threshold(const float2* blurred, const LevelAcc* acc, long long n, int batch,
                          int method, float threshold, std::uint8_t* support, cudaStream_t stream) {
  threshold_kernel<<<grid(n, batch), kThreads, 0, stream>>>(blurred, acc, n, method, threshold,
                                                           support);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

void detwin(std::uint8_t* support, unsigned long long* moments, Dims3 d, int axis3, int batch,
            cudaStream_t stream) {
  QPB_CHECK(cudaMemsetAsync(moments, 0, 2 * sizeof(unsigned long long) * batch, stream));
  detwin_moment_kernel<<<grid(d.n(), batch), kThreads, 0, stream>>>(support, d, axis3, moments);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
  detwin_apply_kernel<<<grid(d.n(), batch), kThreads, 0, stream>>>(support, d, axis3, moments);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

template <class T>
void roll(const T* in, T* out, Dims3 d, int batch, bool to_fft_order, cudaStream_t stream) {
  auto off = [&](int len) { return to_fft_order ? len / 2 : len - len / 2; };
  roll_kernel<T><<<grid(d.n(), batch), kThreads, 0, stream>>>(in, out, d, off(d.d0), off(d.d1),
                                                              off(d.d2));
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

template void roll<float2>(const float2*, float2*, Dims3, int, bool, cudaStream_t);
template void roll<float>(const float*, float*, Dims3, int, bool, cudaStream_t);
template void roll<std::uint8_t>(const std::uint8_t*, std::uint8_t*, Dims3, int, bool,
                                 cudaStream_t);

void set_coefficients(Ctrl* ctrl, float a, float b, cudaStream_t stream) {
  set_coefficients_kernel<<<1, 1, 0, stream>>>(ctrl, a, b);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

void set_ctrl(Ctrl* ctrl, const Ctrl& value, cudaStream_t stream) {
  set_ctrl_kernel<<<1, 1, 0, stream>>>(ctrl, value);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

void scale_complex(float2* x, long long count, float scale, cudaStream_t stream) {
  scale_complex_kernel<<<grid(count, 1), kThreads, 0, stream>>>(x, count, scale);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

void to_half(const float2* in, void* out, long long count, cudaStream_t stream) {
  to_half_kernel<<<grid(count, 1), kThreads, 0, stream>>>(in, static_cast<__half2*>(out), count);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

void from_half(const void* in, float2* out, long long count, cudaStream_t stream) {
  from_half_kernel<<<grid(count, 1), kThreads, 0, stream>>>(static_cast<const __half2*>(in), out,
                                                             count);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

}  // namespace qpb
