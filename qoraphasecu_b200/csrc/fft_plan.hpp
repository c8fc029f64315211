// Host-side plans for the line FFTs: the radix sequence of each length and its
// twiddle table W_L^k = exp(-2 pi i k / L), computed in FP64 and rounded once
// to FP32 on upload.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <memory>
#include <mutex>
#include <vector>

namespace qpb {

inline constexpr int kMaxStages = 16;
// Largest prime factor a line length may have; such radices run as a direct
// DFT inside a Stockham stage.
inline constexpr int kMaxPrimeRadix = 127;
// Longest line a shared-memory line pass holds.
inline constexpr int kMaxLine = 8192;

struct LinePlan {
  int length = 1;
  int stages = 0;
  int radix[kMaxStages] = {};
  const float2* twiddle = nullptr;  // device, `length` entries
  // device, the stage-major table of the register-resident transform
  // (stage_table.hpp) for lengths that have one, else `twiddle`
  const float2* stage_twiddle = nullptr;
};

// Radix sequence for a line of length `n` (throws InvalidArgument when a prime
// factor exceeds kMaxPrimeRadix or n exceeds kMaxLine).
std::vector<int> factorize(int n);

// Per-device cache of line plans; twiddle tables live until the cache dies.
class PlanCache {
 public:
  PlanCache() = default;
  PlanCache(const PlanCache&) = delete;
  PlanCache& operator=(const PlanCache&) = delete;
  ~PlanCache();

  const LinePlan& get(int length);

  // Device counter of the line-pass CTAs whose bounded wait for their staged
  // inputs gave up (those CTAs wrote nothing), shared by every pass planned
  // from this cache: a solver's own cache makes it per solver. Allocated and
  // zeroed on first use, which must not fall inside a stream capture.
  int* wait_failures();

  // Reads the counter on `stream` after the work enqueued there, clears it
  // when it is set, and returns what it held. Synchronises `stream`.
  int take_wait_failures(cudaStream_t stream);

 private:
  std::mutex mutex_;
  std::map<int, LinePlan> plans_;
  std::vector<void*> allocations_;
  int* failures_ = nullptr;
};

}  // namespace qpb
