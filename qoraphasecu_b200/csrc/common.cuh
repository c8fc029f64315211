// Shared device/host helpers of the B200 phase-retrieval backend.
//
// The point-wise formulas here restate QoraPhaseCU's src/core/pointwise.hpp so
// that the random starting phases are bit-identical to the reference's CPU
// path and the update coefficients round the same way.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#define QPB_HD __host__ __device__ __forceinline__

namespace qpb {

// src/core/pointwise.hpp:16-17
inline constexpr float kEps = 1e-12f;
inline constexpr float kTwoPi = 6.28318530717958647692f;

// splitmix64 finaliser, src/core/pointwise.hpp:19-24.
QPB_HD std::uint64_t mix64(std::uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Counter-based uniform in [0, 1), src/core/pointwise.hpp:29-32: element
// `index` of start `start` is drawn independently of every other element.
QPB_HD float uniform(std::uint64_t seed, std::uint64_t start, std::uint64_t index) {
  const std::uint64_t key = mix64(seed ^ mix64(start + 1));
  return static_cast<float>(mix64(key + index) >> 40) * 0x1p-24f;
}

// x <- S ? P : a x + b P outside; (a, b) per algorithm, src/core/pointwise.hpp:36-45.
struct Coefficients {
  float a;
  float b;
};

inline Coefficients er_coefficients() { return {0.0f, 0.0f}; }
inline Coefficients hio_coefficients(float beta) { return {1.0f, -beta}; }
inline Coefficients raar_coefficients(float beta) { return {beta, 1.0f - 2.0f * beta}; }

// Signed frequency of FFT-order index k on an axis of length n, pointwise.hpp:48-51.
QPB_HD float fftfreq(std::uint32_t k, std::uint32_t n) {
  const int s = k < (n + 1) / 2 ? static_cast<int>(k) : static_cast<int>(k) - static_cast<int>(n);
  return static_cast<float>(s) / static_cast<float>(n);
}

// ---------------------------------------------------------------- complex
QPB_HD float2 cadd(float2 a, float2 b) { return {a.x + b.x, a.y + b.y}; }
QPB_HD float2 csub(float2 a, float2 b) { return {a.x - b.x, a.y - b.y}; }
QPB_HD float2 cscale(float2 a, float s) { return {a.x * s, a.y * s}; }
QPB_HD float2 cmul(float2 a, float2 b) { return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
// a * conj(b)
QPB_HD float2 cmulc(float2 a, float2 b) { return {a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y}; }
// a * (-i) and a * (+i)
QPB_HD float2 mul_mi(float2 a) { return {a.y, -a.x}; }
QPB_HD float2 mul_pi(float2 a) { return {-a.y, a.x}; }

// ---------------------------------------------------------------- errors
// Status codes of the C ABI (include/qpb.h).
enum Status : int { kOk = 0, kInvalidArgument = 1, kRuntimeError = 2, kTimeout = 3 };

struct InvalidArgument : std::invalid_argument {
  using std::invalid_argument::invalid_argument;
};

// A kernel's bounded wait gave up (QPB_TIMEOUT at the C ABI).
struct Timeout : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void cuda_check(cudaError_t status, const char* what) {
  if (status != cudaSuccess) {
    // A non-sticky failure (an allocation, an invalid argument) stays the
    // thread's last error; clear it so that a later launch check on this
    // thread does not report it again.
    (void)cudaGetLastError();
    throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(status));
  }
}

#define QPB_CHECK(expr) ::qpb::cuda_check((expr), #expr)

// Kernels this library has launched in this process (graph replays count
// every kernel node they run).
void count_launches(unsigned long long n);
unsigned long long launches();

// The thread-local message qpb_last_error() returns.
void set_last_error(const char* message);
void clear_last_error();

// Host-side trace to stderr when the environment sets QPB_TRACE=1.
bool tracing();
void trace(const char* fmt, ...) __attribute__((format(printf, 1, 2)));

}  // namespace qpb
