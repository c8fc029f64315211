// TEST INFRASTRUCTURE (oracle). Binds the reference's existing Backend::cuda
// factory slot to the B200 adapter (qoraphasecu_b200/adapter/b200_solver.cpp),
// in place of src/cpu/no_cuda.cpp, so that the reference's own make_solver,
// reconstruct and best_index (src/core/solver.cpp:61-103), compiled unchanged
// from its sources, reach the B200 backend with Options::backend = cuda. The
// reference's own CUDA backend (src/cuda) is not part of this library. A
// maintainer would add Backend::b200 instead; the adapter is the same.
//
// The other entry points no_cuda.cpp provides (cuda_available,
// cuda_device_info, the qpcu::cuda single operators, operators.hpp:25-33)
// forward to the matching libqpb.so calls.

#include <cstdint>
#include <span>
#include <stdexcept>
#include <vector>

#include "../src/core/backends.hpp"
#include "qoraphasecu/operators.hpp"
#include "qpb.h"

namespace qpcu {

namespace detail {
std::unique_ptr<Solver> make_b200_solver(const Problem& problem, const Options& options);

std::unique_ptr<Solver> make_cuda_solver(const Problem& problem, const Options& options) {
  return make_b200_solver(problem, options);
}
}  // namespace detail

namespace {
void check(qpb_status status) {
  if (status == QPB_OK) return;
  if (status == QPB_INVALID_ARGUMENT) throw std::invalid_argument(qpb_last_error());
  throw std::runtime_error(qpb_last_error());
}
}  // namespace

bool cuda_available() { return qpb_cuda_available() != 0; }

DeviceInfo cuda_device_info() {
  DeviceInfo info;
  char name[256] = {};
  check(qpb_device_info(name, sizeof(name), &info.sm_major, &info.sm_minor, &info.memory_bytes,
                        &info.l2_bytes, &info.peak_bandwidth_gbs));
  info.name = name;
  return info;
}

namespace cuda {

float modulus_project(const Problem& problem, std::span<Complex> obj) {
  qpb_problem p{};
  p.ndim = static_cast<int>(problem.shape.size());
  for (std::size_t a = 0; a < problem.shape.size() && a < 3; ++a) {
    p.shape[a] = static_cast<int64_t>(problem.shape[a]);
  }
  p.amplitude = problem.amplitude.data();
  p.mask = problem.mask.data();
  p.support = problem.support.data();
  float err = 0.0f;
  check(qpb_modulus_project(&p, reinterpret_cast<float*>(obj.data()), QPB_AMP_F32, &err));
  return err;
}

void support_project(std::span<const std::uint8_t> support, std::span<Complex> obj) {
  check(qpb_support_project(support.data(), reinterpret_cast<float*>(obj.data()), obj.size()));
}

std::vector<float> gaussian_blur(std::span<const float> image, const Shape& shape, float sigma) {
  int64_t s[3] = {0, 0, 0};
  for (std::size_t a = 0; a < shape.size() && a < 3; ++a) s[a] = static_cast<int64_t>(shape[a]);
  std::vector<float> out(image.size());
  check(qpb_gaussian_blur(image.data(), static_cast<int>(shape.size()), s, sigma, out.data()));
  return out;
}

}  // namespace cuda

}  // namespace qpcu
