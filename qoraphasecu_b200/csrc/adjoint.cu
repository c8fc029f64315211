// The amplitude loss L(x) = sum over usable pixels of (|F x| - A)^2 (F the
// unitary FFT) and its gradient, for gradient-based reconstruction.
//
// The gradient in PyTorch's convention (dL/dRe x + i dL/dIm x) is
// 2 F^H[(|y| - A) y / |y|], y = F x, which equals 2 (x - P_M x) with the
// reference's modulus projection P_M (src/cpu/kernels.cpp:25-42) up to its
// eps. It is computed by the same fused line passes as a modulus projection:
// forward transform, the gradient's point-wise step with the loss sum on the
// outer axis, inverse transform.

#include <algorithm>
#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/qpb.h"
#include "solver.hpp"

namespace qpb {

namespace {

// Line plans, a control block and a zero counter per device, created on the
// first call and kept for the process.
struct AdjointResources {
  PlanCache plans;
  DeviceBuffer<Ctrl> ctrl{1};
  DeviceBuffer<int> counter{1};
};

AdjointResources& resources() {
  static std::mutex mutex;
  static std::map<int, std::unique_ptr<AdjointResources>> per_device;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  auto& slot = per_device[device];
  if (!slot) slot = std::make_unique<AdjointResources>();
  return *slot;
}

// Every loss becomes NaN when a line pass of this call gave up a bounded wait
// (its CTAs wrote nothing, so the gradient is not valid); the counter is
// cleared for the next call.
__global__ void flag_failures_kernel(int* failures, double* loss, int batch) {
  const bool failed = *failures != 0;
  __syncthreads();
  if (failed) {
    for (int b = threadIdx.x; b < batch; b += blockDim.x) loss[b] = __longlong_as_double(0x7ff8000000000000LL);
    if (threadIdx.x == 0) *failures = 0;
  }
}

void require_aligned(const void* ptr, std::uintptr_t bytes, const char* name) {
  if (reinterpret_cast<std::uintptr_t>(ptr) % bytes != 0) {
    throw InvalidArgument(std::string("qpb_amplitude_loss_grad: ") + name + " must be " +
                          std::to_string(bytes) + "-byte aligned");
  }
}

}  // namespace

void amplitude_loss_grad(int ndim, const long long* shape, int batch, const float* signed_amp,
                         const float2* x, float2* grad, double* loss, cudaStream_t stream) {
  if (batch < 1) throw InvalidArgument("batch must be >= 1");
  // x, grad and the amplitude are moved by bulk copies, which start on
  // 16-byte boundaries.
  require_aligned(x, 16, "x");
  require_aligned(grad, 16, "grad");
  require_aligned(signed_amp, 16, "signed_amplitude");
  require_aligned(loss, alignof(double), "loss");
  ProblemView view;
  view.ndim = ndim;
  for (int a = 0; a < ndim && a < 3; ++a) view.shape[a] = shape[a];
  const Dims3 d = dims_of(view);
  AdjointResources& r = resources();
  PassRunner runner(d, ndim, r.plans);
  QPB_CHECK(cudaMemsetAsync(r.counter.get(), 0, sizeof(int), stream));
  QPB_CHECK(cudaMemsetAsync(loss, 0, sizeof(double) * batch, stream));
  set_ctrl(r.ctrl.get(), Ctrl{loss, 1, 0.0f, 0.0f, r.counter.get()}, stream);
  auto params = [&](Mode m, int axis3) {
    PassParams p = runner.params(m, axis3, batch);
    p.w = grad;
    p.x = const_cast<float2*>(x);
    p.amp = signed_amp;
    p.ctrl = r.ctrl.get();
    p.starts_total = batch;
    p.amp_storage = AmpStorage::kF32;
    return p;
  };
  const int outer = runner.outer();
  runner.launch(Mode::kFwdFromX, 2, params(Mode::kFwdFromX, 2), stream);
  if (runner.has_mid()) runner.launch(Mode::kFwd, 1, params(Mode::kFwd, 1), stream);
  runner.launch(Mode::kGrad, outer, params(Mode::kGrad, outer), stream);
  if (runner.has_mid()) runner.launch(Mode::kInv, 1, params(Mode::kInv, 1), stream);
  runner.launch(Mode::kInv, 2, params(Mode::kInv, 2), stream);
  flag_failures_kernel<<<1, 32, 0, stream>>>(r.plans.wait_failures(), loss, batch);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

namespace {

// One element of the projection after an optimiser step: 0 outside the
// support; inside it, a magnitude above `bound` scaled down onto it.
__device__ __forceinline__ float2 onto_support_and_disc(float2 v, unsigned char inside,
                                                       float bound) {
  if (!inside) return make_float2(0.0f, 0.0f);
  const float m = hypotf(v.x, v.y);
  if (m > bound) {
    const float f = bound / m;
    return make_float2(v.x * f, v.y * f);
  }
  return v;
}

// Two elements a thread per step (one 16-byte load and store), object
// blockIdx.y; `pairs` = numel / 2 (numel even).
__global__ void support_bound_pairs_kernel(float4* x, const uchar2* support, long long pairs,
                                           float bound) {
  float4* obj = x + static_cast<long long>(blockIdx.y) * pairs;
  const long long step = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < pairs;
       i += step) {
    const float4 v = obj[i];
    const uchar2 in = support[i];
    const float2 a = onto_support_and_disc(make_float2(v.x, v.y), in.x, bound);
    const float2 b = onto_support_and_disc(make_float2(v.z, v.w), in.y, bound);
    obj[i] = make_float4(a.x, a.y, b.x, b.y);
  }
}

// One element a thread per step (odd numel or x not 16-byte aligned).
__global__ void support_bound_kernel(float2* x, const unsigned char* support, long long numel,
                                     float bound) {
  float2* obj = x + static_cast<long long>(blockIdx.y) * numel;
  const long long step = static_cast<long long>(gridDim.x) * blockDim.x;
  for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < numel;
       i += step) {
    obj[i] = onto_support_and_disc(obj[i], support[i], bound);
  }
}

}  // namespace

void project_support_bound(long long numel, int batch, const std::uint8_t* support, float bound,
                           float2* x, cudaStream_t stream) {
  if (numel < 1) throw InvalidArgument("numel must be >= 1");
  if (batch < 1 || batch > 65535) throw InvalidArgument("batch must be in [1, 65535]");
  if (!(bound > 0.0f)) throw InvalidArgument("bound must be > 0 (infinity: no bound)");
  if (reinterpret_cast<std::uintptr_t>(x) % alignof(float2) != 0) {
    throw InvalidArgument("qpb_project_support_bound: x must be 8-byte aligned");
  }
  // A grid-stride loop over each object, about 4 waves of 256-thread CTAs
  // over all objects.
  int device = 0;
  int sms = 0;
  QPB_CHECK(cudaGetDevice(&device));
  QPB_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const bool pairs = numel % 2 == 0 && reinterpret_cast<std::uintptr_t>(x) % 16 == 0 &&
                     reinterpret_cast<std::uintptr_t>(support) % 2 == 0;
  const long long items = pairs ? numel / 2 : numel;
  const long long wanted = (items + 255) / 256;
  const long long cap = std::max<long long>(1, 4LL * 8 * sms / batch);
  const dim3 grid(static_cast<unsigned>(std::min(wanted, cap)), static_cast<unsigned>(batch));
  if (pairs) {
    support_bound_pairs_kernel<<<grid, 256, 0, stream>>>(
        reinterpret_cast<float4*>(x), reinterpret_cast<const uchar2*>(support), items, bound);
  } else {
    support_bound_kernel<<<grid, 256, 0, stream>>>(x, support, numel, bound);
  }
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

}  // namespace qpb

extern "C" qpb_status qpb_project_support_bound(int64_t numel, int batch, const uint8_t* support,
                                                float bound, float* x, void* stream) {
  try {
    qpb::clear_last_error();
    if (!support || !x) throw qpb::InvalidArgument("NULL argument");
    qpb::project_support_bound(numel, batch, support, bound, reinterpret_cast<float2*>(x),
                               static_cast<cudaStream_t>(stream));
    return QPB_OK;
  } catch (const std::invalid_argument& e) {
    qpb::set_last_error(e.what());
    return QPB_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    qpb::set_last_error(e.what());
    return QPB_RUNTIME_ERROR;
  }
}

extern "C" qpb_status qpb_amplitude_loss_grad(int ndim, const int64_t* shape, int batch,
                                              const float* signed_amplitude, const float* x,
                                              float* grad, double* loss, void* stream) {
  try {
    qpb::clear_last_error();
    if (!shape || !signed_amplitude || !x || !grad || !loss) {
      throw qpb::InvalidArgument("NULL argument");
    }
    long long sh[3] = {0, 0, 0};
    for (int a = 0; a < ndim && a < 3; ++a) sh[a] = shape[a];
    qpb::amplitude_loss_grad(ndim, sh, batch, signed_amplitude,
                             reinterpret_cast<const float2*>(x), reinterpret_cast<float2*>(grad),
                             loss, static_cast<cudaStream_t>(stream));
    return QPB_OK;
  } catch (const std::invalid_argument& e) {
    qpb::set_last_error(e.what());
    return QPB_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    qpb::set_last_error(e.what());
    return QPB_RUNTIME_ERROR;
  }
}
