// Scoring and problem set-up on the device: the aligned object error of a
// batch of reconstructions against a reference (src/core/metrics.cpp:17-86)
// and the simulated intensity |centred unitary FFT|^2 (src/core/problem.cpp:90-99).
//
// Aligned error, per candidate b and for both b and its twin conj(b(-r)):
//   F(ref) and F(b) by the line passes, c = IFFT(F(ref) conj(F(b))) (cyclic
//   cross-correlation), s = argmax |c|^2 (the first index on ties, as
//   std::max_element), shifted = b rolled by s, rotation = overlap/|overlap|
//   with overlap = sum ref conj(shifted) in FP64, error =
//   sqrt(sum |rotation shifted - ref|^2 / sum |ref|^2); the result is the
//   smaller of the direct and twin errors.

#include <cfloat>
#include <cmath>
#include <vector>

#include "solver.hpp"

namespace qpb {

namespace {

constexpr int kThreads = 256;

int blocks_for(long long work) {
  return static_cast<int>(std::min<long long>(std::max<long long>((work + kThreads - 1) / kThreads, 1),
                                              148LL * 8));
}

// out[b][z,y,x] = conj(in[b][(-z) mod d0, (-y) mod d1, (-x) mod d2])
__global__ void twin_kernel(const float2* in, float2* out, Dims3 d) {
  const long long n = d.n();
  in += blockIdx.y * n;
  out += blockIdx.y * n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const int x = static_cast<int>(i % d.d2);
    const int y = static_cast<int>((i / d.d2) % d.d1);
    const int z = static_cast<int>(i / (static_cast<long long>(d.d2) * d.d1));
    const long long src = (static_cast<long long>((d.d0 - z) % d.d0) * d.d1 + (d.d1 - y) % d.d1) *
                              d.d2 +
                          (d.d2 - x) % d.d2;
    const float2 v = in[src];
    out[i] = {v.x, -v.y};
  }
}

// c[b][i] = fr[i] * conj(c[b][i])
__global__ void correlate_kernel(const float2* fr, float2* c, long long n) {
  c += blockIdx.y * n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 a = fr[i], b = c[i];
    c[i] = {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y};
  }
}

// key[b] = max over i of (bits(|c|^2) << 32) | (0xffffffff - i): the largest
// |c|^2, the smallest index among equals. |c|^2 >= 0, so its float bits order
// like its value. Indices are below 2^32 (numel <= 2^39 is not reachable: the
// largest shape is 8192 per axis in 2D).
__global__ void argmax_kernel(const float2* c, long long n, unsigned long long* key) {
  c += blockIdx.y * n;
  unsigned long long best = 0;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 v = c[i];
    const float m = v.x * v.x + v.y * v.y;
    const unsigned long long k =
        (static_cast<unsigned long long>(__float_as_uint(m)) << 32) |
        (0xffffffffULL - static_cast<unsigned long long>(i));
    best = k > best ? k : best;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, best, o);
    best = other > best ? other : best;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(key + blockIdx.y, best);
}

__device__ __forceinline__ long long shifted_source(long long i, Dims3 d, long long peak) {
  const long long plane = static_cast<long long>(d.d1) * d.d2;
  const int s0 = static_cast<int>(peak / plane);
  const int s1 = static_cast<int>((peak / d.d2) % d.d1);
  const int s2 = static_cast<int>(peak % d.d2);
  const int x = static_cast<int>(i % d.d2);
  const int y = static_cast<int>((i / d.d2) % d.d1);
  const int z = static_cast<int>(i / plane);
  return (static_cast<long long>((z + d.d0 - s0) % d.d0) * d.d1 + (y + d.d1 - s1) % d.d1) * d.d2 +
         (x + d.d2 - s2) % d.d2;
}

__device__ __forceinline__ double block_sum(double v, double* shared) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) shared[threadIdx.x >> 5] = v;
  __syncthreads();
  double total = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) total += shared[w];
  }
  __syncthreads();
  return total;
}

// acc[b] = {Re, Im of sum ref conj(shifted), sum |ref|^2, sum |rot shifted - ref|^2}.
// pass 0 accumulates the first three; pass 1 the last, with rot from pass 0.
template <int PASS>
__global__ void overlap_kernel(const float2* ref, const float2* cand, Dims3 d,
                               const unsigned long long* key, double* acc) {
  __shared__ double shared[kThreads / 32];
  const long long n = d.n();
  const int b = blockIdx.y;
  cand += b * n;
  double* a = acc + 4 * b;
  const long long peak = static_cast<long long>(0xffffffffULL - (key[b] & 0xffffffffULL));
  double re = 0.0, im = 0.0, norm = 0.0, diff = 0.0;
  double rr = 1.0, ri = 0.0;
  if constexpr (PASS == 1) {
    const double mag = sqrt(a[0] * a[0] + a[1] * a[1]);
    if (mag > 0.0) {
      rr = a[0] / mag;
      ri = a[1] / mag;
    }
  }
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 r = ref[i];
    const float2 s = cand[shifted_source(i, d, peak)];
    if constexpr (PASS == 0) {
      re += static_cast<double>(r.x) * s.x + static_cast<double>(r.y) * s.y;
      im += static_cast<double>(r.y) * s.x - static_cast<double>(r.x) * s.y;
      norm += static_cast<double>(r.x) * r.x + static_cast<double>(r.y) * r.y;
    } else {
      const double dx = rr * s.x - ri * s.y - r.x;
      const double dy = rr * s.y + ri * s.x - r.y;
      diff += dx * dx + dy * dy;
    }
  }
  if constexpr (PASS == 0) {
    re = block_sum(re, shared);
    im = block_sum(im, shared);
    norm = block_sum(norm, shared);
    if (threadIdx.x == 0) {
      atomicAdd(a + 0, re);
      atomicAdd(a + 1, im);
      atomicAdd(a + 2, norm);
    }
  } else {
    diff = block_sum(diff, shared);
    if (threadIdx.x == 0) atomicAdd(a + 3, diff);
  }
}

// out[b][i] = rotation_c * cand[c][shifted_source(i)] for the chosen
// candidate c of object b (its direct form or its twin), rotation_c =
// overlap_c / |overlap_c|: object b moved onto the reference.
__global__ void apply_kernel(const float2* cand, Dims3 d, const unsigned long long* key,
                             const double* acc, const int* choice, float2* out) {
  const long long n = d.n();
  const int b = blockIdx.y;
  const int c = choice[b];
  const float2* src = cand + c * n;
  const double* a = acc + 4 * c;
  const long long peak = static_cast<long long>(0xffffffffULL - (key[c] & 0xffffffffULL));
  const double mag = sqrt(a[0] * a[0] + a[1] * a[1]);
  const float rr = mag > 0.0 ? static_cast<float>(a[0] / mag) : 1.0f;
  const float ri = mag > 0.0 ? static_cast<float>(a[1] / mag) : 0.0f;
  out += b * n;
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 s = src[shifted_source(i, d, peak)];
    out[i] = {rr * s.x - ri * s.y, rr * s.y + ri * s.x};
  }
}

// mean[i] = (1 / batch) sum_b aligned[b][i], summed in order of b.
__global__ void mean_kernel(const float2* aligned, long long n, int batch, float2* mean) {
  const float inv = 1.0f / static_cast<float>(batch);
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    float2 sum = {0.0f, 0.0f};
    for (int b = 0; b < batch; ++b) {
      const float2 v = aligned[b * n + i];
      sum.x += v.x;
      sum.y += v.y;
    }
    mean[i] = {sum.x * inv, sum.y * inv};
  }
}

__global__ void intensity_kernel(const float2* w, float* out, long long n, float scale2) {
  for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<long long>(gridDim.x) * blockDim.x) {
    const float2 v = w[i];
    out[i] = (v.x * v.x + v.y * v.y) * scale2;
  }
}

struct Transforms {
  Dims3 d;
  int ndim;
  PlanCache plans;
  PassRunner runner;
  Transforms(Dims3 dims, int nd) : d(dims), ndim(nd), runner(dims, nd, plans) {}

  // In-place unnormalised transform of `batch` arrays along every axis.
  void run(Mode mode, float2* w, int batch, cudaStream_t s) {
    for (int axis3 = runner.outer(); axis3 < 3; ++axis3) {
      PassParams p = runner.params(mode, axis3, batch);
      p.w = w;
      p.x = w;
      runner.launch(mode, axis3, p, s);
    }
  }
};

ProblemView shape_view(int ndim, const long long* shape) {
  if (ndim != 2 && ndim != 3) {
    throw InvalidArgument("shape must be 2D or 3D, got ndim=" + std::to_string(ndim));
  }
  ProblemView v;
  v.ndim = ndim;
  for (int a = 0; a < ndim; ++a) v.shape[a] = shape[a];
  return v;
}

}  // namespace

void align(const float2* a, const float2* reference, int ndim, const long long* shape, int batch,
           float* errors, float2* aligned, float2* mean) {
  if (batch < 1) throw InvalidArgument("batch must be >= 1");
  const Dims3 d = dims_of(shape_view(ndim, shape));
  const long long n = d.n();
  if (n >= (1LL << 32)) throw InvalidArgument("array too large");
  Transforms t(d, ndim);
  Stream s;
  const int cands = 2 * batch;  // direct candidates, then their twins
  DeviceBuffer<float2> ref(static_cast<std::size_t>(n));
  DeviceBuffer<float2> fr(static_cast<std::size_t>(n));
  DeviceBuffer<float2> cand(static_cast<std::size_t>(cands) * n);
  DeviceBuffer<float2> corr(static_cast<std::size_t>(cands) * n);
  DeviceBuffer<unsigned long long> key(static_cast<std::size_t>(cands));
  DeviceBuffer<double> acc(4 * static_cast<std::size_t>(cands));
  const std::size_t bytes = static_cast<std::size_t>(n) * sizeof(float2);
  QPB_CHECK(cudaMemcpyAsync(ref.get(), reference, bytes, cudaMemcpyHostToDevice, s));
  QPB_CHECK(cudaMemcpyAsync(cand.get(), a, bytes * batch, cudaMemcpyHostToDevice, s));
  QPB_CHECK(cudaMemsetAsync(key.get(), 0, key.size() * sizeof(unsigned long long), s));
  QPB_CHECK(cudaMemsetAsync(acc.get(), 0, acc.size() * sizeof(double), s));
  const dim3 grid_b(static_cast<unsigned>(blocks_for(n)), static_cast<unsigned>(batch));
  const dim3 grid_c(static_cast<unsigned>(blocks_for(n)), static_cast<unsigned>(cands));
  twin_kernel<<<grid_b, kThreads, 0, s>>>(cand.get(), cand.get() + batch * n, d);
  QPB_CHECK(cudaGetLastError());
  QPB_CHECK(cudaMemcpyAsync(fr.get(), ref.get(), bytes, cudaMemcpyDeviceToDevice, s));
  QPB_CHECK(cudaMemcpyAsync(corr.get(), cand.get(), bytes * cands, cudaMemcpyDeviceToDevice, s));
  t.run(Mode::kFwd, fr.get(), 1, s);
  t.run(Mode::kFwd, corr.get(), cands, s);
  correlate_kernel<<<grid_c, kThreads, 0, s>>>(fr.get(), corr.get(), n);
  QPB_CHECK(cudaGetLastError());
  t.run(Mode::kInv, corr.get(), cands, s);
  argmax_kernel<<<grid_c, kThreads, 0, s>>>(corr.get(), n, key.get());
  QPB_CHECK(cudaGetLastError());
  overlap_kernel<0><<<grid_c, kThreads, 0, s>>>(ref.get(), cand.get(), d, key.get(), acc.get());
  QPB_CHECK(cudaGetLastError());
  overlap_kernel<1><<<grid_c, kThreads, 0, s>>>(ref.get(), cand.get(), d, key.get(), acc.get());
  QPB_CHECK(cudaGetLastError());
  count_launches(6);
  std::vector<double> host(acc.size());
  QPB_CHECK(cudaMemcpyAsync(host.data(), acc.get(), host.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, s));
  s.sync();
  check_waits(t.plans, s);
  std::vector<int> choice(static_cast<std::size_t>(batch));
  for (int b = 0; b < batch; ++b) {
    float e[2];
    for (int k = 0; k < 2; ++k) {
      const double* v = host.data() + 4 * (b + k * batch);
      e[k] = static_cast<float>(std::sqrt(v[3] / std::max(v[2], DBL_MIN)));
    }
    choice[b] = e[0] <= e[1] ? b : b + batch;
    if (errors) errors[b] = std::min(e[0], e[1]);
  }
  if (!aligned && !mean) return;
  // The chosen candidate of every object, moved onto the reference, and their mean.
  DeviceBuffer<int> chosen(static_cast<std::size_t>(batch));
  QPB_CHECK(cudaMemcpyAsync(chosen.get(), choice.data(), choice.size() * sizeof(int),
                            cudaMemcpyHostToDevice, s));
  apply_kernel<<<grid_b, kThreads, 0, s>>>(cand.get(), d, key.get(), acc.get(), chosen.get(),
                                          corr.get());
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
  if (mean) {
    mean_kernel<<<blocks_for(n), kThreads, 0, s>>>(corr.get(), n, batch, fr.get());
    QPB_CHECK(cudaGetLastError());
    count_launches(1);
    QPB_CHECK(cudaMemcpyAsync(mean, fr.get(), bytes, cudaMemcpyDeviceToHost, s));
  }
  if (aligned) {
    QPB_CHECK(cudaMemcpyAsync(aligned, corr.get(), bytes * batch, cudaMemcpyDeviceToHost, s));
  }
  s.sync();
}

void aligned_error(const float2* a, const float2* reference, int ndim, const long long* shape,
                   int batch, float* out) {
  align(a, reference, ndim, shape, batch, out, nullptr, nullptr);
}

void simulate_intensity(const float2* object, int ndim, const long long* shape, float* out) {
  const Dims3 d = dims_of(shape_view(ndim, shape));
  const long long n = d.n();
  Transforms t(d, ndim);
  Stream s;
  DeviceBuffer<float2> obj(static_cast<std::size_t>(n));
  DeviceBuffer<float2> w(static_cast<std::size_t>(n));
  DeviceBuffer<float> ordered(static_cast<std::size_t>(n));
  DeviceBuffer<float> centred(static_cast<std::size_t>(n));
  QPB_CHECK(cudaMemcpyAsync(obj.get(), object, static_cast<std::size_t>(n) * sizeof(float2),
                            cudaMemcpyHostToDevice, s));
  roll<float2>(obj.get(), w.get(), d, 1, true, s);
  t.run(Mode::kFwd, w.get(), 1, s);
  intensity_kernel<<<blocks_for(n), kThreads, 0, s>>>(w.get(), ordered.get(), n,
                                                       1.0f / static_cast<float>(n));
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
  roll<float>(ordered.get(), centred.get(), d, 1, false, s);
  QPB_CHECK(cudaMemcpyAsync(out, centred.get(), static_cast<std::size_t>(n) * sizeof(float),
                            cudaMemcpyDeviceToHost, s));
  s.sync();
  check_waits(t.plans, s);
}

}  // namespace qpb
