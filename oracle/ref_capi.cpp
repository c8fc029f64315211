// TEST INFRASTRUCTURE (oracle). A C wrapper over the reference's own public
// C++ API (include/qoraphasecu/*.hpp), compiled together with its CPU sources
// into oracle/_ref/libqpcu_ref.so so that tests and the CPU baseline can call
// the unmodified CpuSolver from Python. Nothing here re-implements an
// algorithm: every call forwards to the reference.

#include <omp.h>

#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../src/cpu/fft.hpp"
#include "qoraphasecu/qoraphasecu.hpp"

namespace {

thread_local std::string g_error;

template <class F>
int guarded(F&& f) {
  try {
    g_error.clear();
    f();
    return 0;
  } catch (const std::invalid_argument& e) {
    g_error = e.what();
    return 1;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}

qpcu::Shape shape_of(int ndim, const int64_t* shape) {
  qpcu::Shape s;
  for (int a = 0; a < ndim; ++a) s.push_back(static_cast<std::size_t>(shape[a]));
  return s;
}

struct Op {
  int kind, n;
  float beta, threshold, sigma;
  int method, axis;
};

qpcu::Recipe recipe_of(const Op* ops, std::size_t count) {
  qpcu::Recipe r;
  for (std::size_t i = 0; i < count; ++i) {
    const Op& o = ops[i];
    switch (o.kind) {
      case 0: r.ops.emplace_back(qpcu::ER{o.n}); break;
      case 1: r.ops.emplace_back(qpcu::HIO{o.n, o.beta}); break;
      case 2: r.ops.emplace_back(qpcu::RAAR{o.n, o.beta}); break;
      case 3:
        r.ops.emplace_back(qpcu::Shrinkwrap{o.threshold, o.sigma,
                                            o.method ? qpcu::Threshold::rms : qpcu::Threshold::max});
        break;
      case 4: r.ops.emplace_back(qpcu::DetwinBegin{o.axis}); break;
      case 5: r.ops.emplace_back(qpcu::DetwinEnd{}); break;
      default: throw std::invalid_argument("unknown op");
    }
  }
  return r;
}

qpcu::Problem problem_of(const float* amp, const uint8_t* mask, const uint8_t* support, int ndim,
                         const int64_t* shape) {
  const qpcu::Shape s = shape_of(ndim, shape);
  const std::size_t n = qpcu::numel(s);
  return qpcu::Problem{s, std::vector<float>(amp, amp + n), std::vector<std::uint8_t>(mask, mask + n),
                       std::vector<std::uint8_t>(support, support + n)};
}

struct RefSolver {
  qpcu::Shape shape;
  std::unique_ptr<qpcu::Solver> solver;
};

}  // namespace

extern "C" {

const char* qref_last_error(void) { return g_error.c_str(); }

void qref_set_threads(int threads) { omp_set_num_threads(threads); }

int qref_fft(const float* in, float* out, int ndim, const int64_t* shape, int forward) {
  return guarded([&] {
    const qpcu::Shape s = shape_of(ndim, shape);
    const std::size_t n = qpcu::numel(s);
    const auto* src = reinterpret_cast<const qpcu::Complex*>(in);
    auto* dst = reinterpret_cast<qpcu::Complex*>(out);
    qpcu::cpu::Fft fft(s);
    if (forward) {
      fft.forward({src, n}, {dst, n});
    } else {
      fft.inverse({src, n}, {dst, n});
    }
  });
}

int qref_make_problem(const float* intensity, int ndim, const int64_t* shape, const uint8_t* support,
                      const uint8_t* mask, float threshold, float* amp_out, uint8_t* mask_out,
                      uint8_t* support_out) {
  return guarded([&] {
    const qpcu::Shape s = shape_of(ndim, shape);
    const std::size_t n = ndim > 0 ? qpcu::numel(s) : 0;
    const auto p = qpcu::make_problem({intensity, n}, s,
                                      support ? std::span<const uint8_t>(support, n)
                                              : std::span<const uint8_t>{},
                                      mask ? std::span<const uint8_t>(mask, n)
                                           : std::span<const uint8_t>{},
                                      threshold);
    std::memcpy(amp_out, p.amplitude.data(), n * sizeof(float));
    std::memcpy(mask_out, p.mask.data(), n);
    std::memcpy(support_out, p.support.data(), n);
  });
}

int qref_modulus_project(const float* amp, const uint8_t* mask, const uint8_t* support, int ndim,
                         const int64_t* shape, float* obj, float* err) {
  return guarded([&] {
    const auto p = problem_of(amp, mask, support, ndim, shape);
    *err = qpcu::cpu::modulus_project(
        p, {reinterpret_cast<qpcu::Complex*>(obj), qpcu::numel(p.shape)});
  });
}

int qref_gaussian_blur(const float* image, int ndim, const int64_t* shape, float sigma, float* out) {
  return guarded([&] {
    const qpcu::Shape s = shape_of(ndim, shape);
    const auto r = qpcu::cpu::gaussian_blur({image, qpcu::numel(s)}, s, sigma);
    std::memcpy(out, r.data(), r.size() * sizeof(float));
  });
}

int qref_half_support(const uint8_t* support, int ndim, const int64_t* shape, int axis,
                      uint8_t* out) {
  return guarded([&] {
    const qpcu::Shape s = shape_of(ndim, shape);
    const auto r = qpcu::half_support({support, qpcu::numel(s)}, s, axis);
    std::memcpy(out, r.data(), r.size());
  });
}

int qref_autocorrelation_support(const float* intensity, int ndim, const int64_t* shape,
                                 float threshold, uint8_t* out) {
  return guarded([&] {
    const qpcu::Shape s = shape_of(ndim, shape);
    const auto r = qpcu::autocorrelation_support({intensity, qpcu::numel(s)}, s, threshold);
    std::memcpy(out, r.data(), r.size());
  });
}

int qref_simulate_intensity(const float* obj, int ndim, const int64_t* shape, float* out) {
  return guarded([&] {
    const qpcu::Shape s = shape_of(ndim, shape);
    const auto r = qpcu::simulate_intensity(
        {reinterpret_cast<const qpcu::Complex*>(obj), qpcu::numel(s)}, s);
    std::memcpy(out, r.data(), r.size() * sizeof(float));
  });
}

int qref_aligned_error(const float* a, const float* ref, int ndim, const int64_t* shape,
                       float* out) {
  return guarded([&] {
    const qpcu::Shape s = shape_of(ndim, shape);
    const std::size_t n = qpcu::numel(s);
    *out = qpcu::aligned_error({reinterpret_cast<const qpcu::Complex*>(a), n},
                               {reinterpret_cast<const qpcu::Complex*>(ref), n}, s);
  });
}

int qref_create(const float* amp, const uint8_t* mask, const uint8_t* support, int ndim,
                const int64_t* shape, int starts, uint64_t seed, const float* start,
                int sync_every, void** out) {
  return guarded([&] {
    auto p = problem_of(amp, mask, support, ndim, shape);
    qpcu::Options o;
    o.backend = qpcu::Backend::cpu;
    o.starts = starts;
    o.seed = seed;
    o.sync_every = sync_every;
    if (start) {
      const auto* c = reinterpret_cast<const qpcu::Complex*>(start);
      o.start.assign(c, c + qpcu::numel(p.shape) * static_cast<std::size_t>(starts));
    }
    auto* r = new RefSolver{p.shape, qpcu::make_solver(p, o)};
    *out = r;
  });
}

// qref_create with the backend (0 cpu, 1 cuda: whatever the library binds
// there), the variant (qpcu::Variant, used by the reference's CUDA backend)
// and the starts per batched plan.
int qref_create_backend(const float* amp, const uint8_t* mask, const uint8_t* support, int ndim,
                        const int64_t* shape, int starts, uint64_t seed, const float* start,
                        int sync_every, int backend, int variant, int batch, void** out) {
  return guarded([&] {
    auto p = problem_of(amp, mask, support, ndim, shape);
    qpcu::Options o;
    o.backend = backend == 1 ? qpcu::Backend::cuda : qpcu::Backend::cpu;
    o.variant = static_cast<qpcu::Variant>(variant);
    o.batch = batch;
    o.starts = starts;
    o.seed = seed;
    o.sync_every = sync_every;
    if (start) {
      const auto* c = reinterpret_cast<const qpcu::Complex*>(start);
      o.start.assign(c, c + qpcu::numel(p.shape) * static_cast<std::size_t>(starts));
    }
    auto* r = new RefSolver{p.shape, qpcu::make_solver(p, o)};
    *out = r;
  });
}

// qpcu::reconstruct (src/core/solver.cpp:88-93) and qpcu::best_index
// (:95-103) through the reference's public API on a made problem; outputs as
// qref_results, *best the index best_index picks.
int qref_reconstruct(const float* amp, const uint8_t* mask, const uint8_t* support, int ndim,
                     const int64_t* shape, const void* ops, size_t count, int starts, uint64_t seed,
                     int backend, float* objects, uint8_t* supports, float* errors, int* best) {
  return guarded([&] {
    const auto p = problem_of(amp, mask, support, ndim, shape);
    qpcu::Options o;
    o.backend = backend == 1 ? qpcu::Backend::cuda : qpcu::Backend::cpu;
    o.starts = starts;
    o.seed = seed;
    const auto runs = qpcu::reconstruct(p, recipe_of(static_cast<const Op*>(ops), count), o);
    const std::size_t n = qpcu::numel(p.shape);
    for (std::size_t s = 0; s < runs.size(); ++s) {
      if (objects) std::memcpy(objects + 2 * s * n, runs[s].object.data(), n * sizeof(qpcu::Complex));
      if (supports) std::memcpy(supports + s * n, runs[s].support.data(), n);
      if (errors) {
        std::memcpy(errors + s * runs[s].errors.size(), runs[s].errors.data(),
                    runs[s].errors.size() * sizeof(float));
      }
    }
    *best = static_cast<int>(qpcu::best_index(runs));
  });
}

// qpcu::cuda_available (solver.hpp:85) of the library's build.
int qref_cuda_available(void) { return qpcu::cuda_available() ? 1 : 0; }

int qref_run(void* solver, const void* ops, size_t count) {
  return guarded([&] {
    static_cast<RefSolver*>(solver)->solver->run(recipe_of(static_cast<const Op*>(ops), count));
  });
}

int qref_results(void* solver, float* objects, uint8_t* supports, float* errors, size_t* count) {
  return guarded([&] {
    const auto runs = static_cast<RefSolver*>(solver)->solver->results();
    const std::size_t n = qpcu::numel(static_cast<RefSolver*>(solver)->shape);
    *count = runs.empty() ? 0 : runs[0].errors.size();
    for (std::size_t s = 0; s < runs.size(); ++s) {
      if (objects) std::memcpy(objects + 2 * s * n, runs[s].object.data(), n * sizeof(qpcu::Complex));
      if (supports) std::memcpy(supports + s * n, runs[s].support.data(), n);
      if (errors) {
        std::memcpy(errors + s * runs[s].errors.size(), runs[s].errors.data(),
                    runs[s].errors.size() * sizeof(float));
      }
    }
  });
}

size_t qref_error_count(void* solver) {
  const auto runs = static_cast<RefSolver*>(solver)->solver->results();
  return runs.empty() ? 0 : runs[0].errors.size();
}

void qref_destroy(void* solver) { delete static_cast<RefSolver*>(solver); }

}  // extern "C"
