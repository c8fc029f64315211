#include "fft_plan.hpp"

#include <cmath>
#include <string>

#include "common.cuh"
#include "stage_table.hpp"

namespace qpb {

std::vector<int> factorize(int n) {
  if (n < 1) throw InvalidArgument("line length must be >= 1");
  if (n > kMaxLine) {
    throw InvalidArgument("axis length " + std::to_string(n) + " exceeds the supported maximum " +
                          std::to_string(kMaxLine));
  }
  std::vector<int> radices;
  int rest = n;
  // Fewest Stockham stages first: radix 8, then 4, then 2 for the power of two.
  while (rest % 8 == 0) {
    radices.push_back(8);
    rest /= 8;
  }
  if (rest % 4 == 0) {
    radices.push_back(4);
    rest /= 4;
  }
  if (rest % 2 == 0) {
    radices.push_back(2);
    rest /= 2;
  }
  for (int p = 3; rest > 1; p += 2) {
    while (rest % p == 0) {
      if (p > kMaxPrimeRadix) {
        throw InvalidArgument("axis length " + std::to_string(n) + " has the prime factor " +
                              std::to_string(p) + " > " + std::to_string(kMaxPrimeRadix));
      }
      radices.push_back(p);
      rest /= p;
    }
  }
  if (static_cast<int>(radices.size()) > kMaxStages) {
    throw InvalidArgument("axis length " + std::to_string(n) + " needs too many FFT stages");
  }
  return radices;
}

PlanCache::~PlanCache() {
  for (void* p : allocations_) cudaFree(p);
}

int* PlanCache::wait_failures() {
  std::lock_guard<std::mutex> lock(mutex_);
  if (!failures_) {
    void* dev = nullptr;
    QPB_CHECK(cudaMalloc(&dev, sizeof(int)));
    allocations_.push_back(dev);
    QPB_CHECK(cudaMemset(dev, 0, sizeof(int)));
    failures_ = static_cast<int*>(dev);
  }
  return failures_;
}

int PlanCache::take_wait_failures(cudaStream_t stream) {
  int* counter = wait_failures();
  int failures = 0;
  QPB_CHECK(cudaMemcpyAsync(&failures, counter, sizeof(int), cudaMemcpyDeviceToHost, stream));
  QPB_CHECK(cudaStreamSynchronize(stream));
  if (failures) {
    QPB_CHECK(cudaMemsetAsync(counter, 0, sizeof(int), stream));
    QPB_CHECK(cudaStreamSynchronize(stream));
  }
  return failures;
}

const LinePlan& PlanCache::get(int length) {
  std::lock_guard<std::mutex> lock(mutex_);
  if (auto it = plans_.find(length); it != plans_.end()) return it->second;
  LinePlan plan;
  plan.length = length;
  const auto radices = factorize(length);
  plan.stages = static_cast<int>(radices.size());
  for (int s = 0; s < plan.stages; ++s) plan.radix[s] = radices[s];
  std::vector<float2> host(static_cast<std::size_t>(length));
  for (int k = 0; k < length; ++k) {
    // exp(-2 pi i k / L) in double, rounded once.
    const double angle = -2.0 * M_PI * static_cast<double>(k) / static_cast<double>(length);
    host[k] = {static_cast<float>(std::cos(angle)), static_cast<float>(std::sin(angle))};
  }
  // The stage-major table holds entries of the same W_L^e, so both tables
  // carry identical values.
  const StageGeometry g = stage_geometry(length);
  for (int i = 0; i < g.count; ++i) host.push_back(host[stage_twiddle_exponent(g, length, i)]);
  void* dev = nullptr;
  QPB_CHECK(cudaMalloc(&dev, host.size() * sizeof(float2)));
  allocations_.push_back(dev);
  QPB_CHECK(cudaMemcpy(dev, host.data(), host.size() * sizeof(float2), cudaMemcpyHostToDevice));
  plan.twiddle = static_cast<const float2*>(dev);
  plan.stage_twiddle = g.count > 0 ? plan.twiddle + length : plan.twiddle;
  return plans_.emplace(length, plan).first->second;
}

}  // namespace qpb
