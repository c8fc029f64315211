// extern "C" boundary of libqpb.so (include/qpb.h). Exceptions are caught here
// and turned into status codes plus a thread-local message.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

#include "../../include/qpb.h"
#include "batch.hpp"
#include "device_setup.cuh"
#include "solver.hpp"

struct qpb_solver {
  qpb::BatchSolver impl;
  qpb_solver(const std::vector<qpb::ProblemView>& p, const qpb::SolverOptions& o) : impl(p, o) {}
};

namespace {

thread_local std::string g_last_error;

template <class F>
qpb_status guarded(F&& f) {
  try {
    g_last_error.clear();
    f();
    return QPB_OK;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return QPB_INVALID_ARGUMENT;
  } catch (const qpb::Timeout& e) {
    g_last_error = e.what();
    return QPB_TIMEOUT;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return QPB_RUNTIME_ERROR;
  } catch (...) {
    g_last_error = "unknown error";
    return QPB_RUNTIME_ERROR;
  }
}

void require(bool ok, const char* what) {
  if (!ok) throw qpb::InvalidArgument(what);
}

qpb::ProblemView view(const qpb_problem* p) {
  require(p != nullptr, "problem is NULL");
  qpb::ProblemView v;
  v.ndim = p->ndim;
  for (int a = 0; a < 3; ++a) v.shape[a] = a < p->ndim ? p->shape[a] : 0;
  v.amplitude = p->amplitude;
  v.mask = p->mask;
  v.support = p->support;
  return v;
}

long long numel_checked(int ndim, const int64_t* shape) {
  require(shape != nullptr, "shape is NULL");
  if (ndim != 2 && ndim != 3) {
    throw qpb::InvalidArgument("shape must be 2D or 3D, got ndim=" + std::to_string(ndim));
  }
  long long n = 1;
  for (int a = 0; a < ndim; ++a) {
    if (shape[a] <= 0) throw qpb::InvalidArgument("shape has a zero-length axis");
    n *= shape[a];
  }
  return n;
}

qpb::AmpStorage storage_of(int s) {
  if (s < 0 || s > 2) throw qpb::InvalidArgument("unknown amplitude storage");
  return static_cast<qpb::AmpStorage>(s);
}

// The runtime's current device is per host thread: make the solver's current.
void use_solver_device(const qpb_solver* solver) {
  QPB_CHECK(cudaSetDevice(solver->impl.device()));
}

// Device arrays a caller lends must be aligned to their element type.
void require_aligned(const void* ptr, std::size_t bytes, const char* name) {
  if (reinterpret_cast<std::uintptr_t>(ptr) % bytes != 0) {
    throw qpb::InvalidArgument(std::string(name) + " must be " + std::to_string(bytes) +
                               "-byte aligned");
  }
}

}  // namespace

namespace qpb {
void set_last_error(const char* message) { g_last_error = message; }
void clear_last_error() { g_last_error.clear(); }
}  // namespace qpb

extern "C" {

const char* qpb_last_error(void) { return g_last_error.c_str(); }

int qpb_cuda_available(void) {
  int count = 0;
  return cudaGetDeviceCount(&count) == cudaSuccess && count > 0;
}

qpb_status qpb_set_device(int device) {
  return guarded([&] { QPB_CHECK(cudaSetDevice(device)); });
}

qpb_status qpb_device_info(char* name_out, size_t name_len, int* sm_major, int* sm_minor,
                           size_t* memory_bytes, size_t* l2_bytes, double* peak_bandwidth_gbs) {
  return guarded([&] {
    if (!qpb_cuda_available()) throw std::runtime_error("no CUDA device available");
    int device = 0;
    QPB_CHECK(cudaGetDevice(&device));
    cudaDeviceProp prop{};
    QPB_CHECK(cudaGetDeviceProperties(&prop, device));
    int clock_khz = 0;
    QPB_CHECK(cudaDeviceGetAttribute(&clock_khz, cudaDevAttrMemoryClockRate, device));
    if (name_out && name_len) {
      std::strncpy(name_out, prop.name, name_len - 1);
      name_out[name_len - 1] = '\0';
    }
    if (sm_major) *sm_major = prop.major;
    if (sm_minor) *sm_minor = prop.minor;
    if (memory_bytes) *memory_bytes = prop.totalGlobalMem;
    if (l2_bytes) *l2_bytes = static_cast<size_t>(prop.l2CacheSize);
    // Double data rate over the bus (operators.cu:18-36 of the reference).
    if (peak_bandwidth_gbs) {
      *peak_bandwidth_gbs = 2.0 * clock_khz * 1e3 * (prop.memoryBusWidth / 8.0) / 1e9;
    }
  });
}

qpb_status qpb_make_problem(const float* intensity, int ndim, const int64_t* shape,
                            const uint8_t* support, const uint8_t* mask, float support_threshold,
                            float* amplitude_out, uint8_t* mask_out, uint8_t* support_out) {
  return guarded([&] {
    const long long n = numel_checked(ndim, shape);
    require(intensity && amplitude_out && mask_out && support_out, "NULL array");
    for (long long i = 0; i < n; ++i) {
      if (!std::isfinite(intensity[i])) throw qpb::InvalidArgument("intensity contains NaN or Inf");
    }
    if (mask) {
      bool all_bad = true;
      for (long long i = 0; i < n && all_bad; ++i) all_bad = mask[i] != 0;
      if (all_bad) throw qpb::InvalidArgument("mask marks every pixel as bad; nothing left to fit");
    }
    long long sh[3] = {0, 0, 0};
    for (int a = 0; a < ndim; ++a) sh[a] = shape[a];
    if (support) {
      for (long long i = 0; i < n; ++i) support_out[i] = support[i] != 0;
    } else {
      qpb::autocorrelation_support_host(intensity, ndim, sh, support_threshold, support_out);
    }
    for (long long i = 0; i < n; ++i) {
      amplitude_out[i] = std::sqrt(std::max(intensity[i], 0.0f));
      mask_out[i] = mask ? mask[i] != 0 : 0;
    }
  });
}

qpb_status qpb_autocorrelation_support(const float* intensity, int ndim, const int64_t* shape,
                                       float threshold, uint8_t* out) {
  return guarded([&] {
    numel_checked(ndim, shape);
    require(intensity && out, "NULL array");
    long long sh[3] = {0, 0, 0};
    for (int a = 0; a < ndim; ++a) sh[a] = shape[a];
    qpb::autocorrelation_support_host(intensity, ndim, sh, threshold, out);
  });
}

qpb_status qpb_half_support(const uint8_t* support, int ndim, const int64_t* shape, int axis,
                            uint8_t* out) {
  return guarded([&] {
    numel_checked(ndim, shape);
    require(support && out, "NULL array");
    long long sh[3] = {0, 0, 0};
    for (int a = 0; a < ndim; ++a) sh[a] = shape[a];
    qpb::half_support(support, ndim, sh, axis, out);
  });
}

namespace {

// The reference's make_solver checks (solver.cpp:61-78), made before any device work.
qpb::SolverOptions options_of(const qpb_options* options) {
  require(options != nullptr, "options is NULL");
  if (options->starts < 1) throw qpb::InvalidArgument("starts must be >= 1");
  if (options->sync_every < 1) throw qpb::InvalidArgument("sync_every must be >= 1");
  if (options->batch < 0 || (options->batch > 0 && options->starts % options->batch != 0)) {
    throw qpb::InvalidArgument("batch must divide starts");
  }
  if (options->variant < QPB_VARIANT_BATCHED || options->variant > QPB_VARIANT_MIXED) {
    throw qpb::InvalidArgument("unknown variant");
  }
  if (options->schedule < QPB_SCHEDULE_AUTO || options->schedule > QPB_SCHEDULE_PERSISTENT) {
    throw qpb::InvalidArgument("unknown schedule");
  }
  qpb::SolverOptions o;
  o.starts = options->starts;
  o.batch = options->batch;
  o.seed = options->seed;
  o.start = reinterpret_cast<const float2*>(options->start);
  o.sync_every = options->sync_every;
  o.variant = static_cast<qpb::Variant>(options->variant);
  o.amp_storage = storage_of(options->amp_storage);
  o.device = options->device;
  o.stream = static_cast<cudaStream_t>(options->stream);
  o.schedule = static_cast<qpb::Schedule>(options->schedule);
  return o;
}

qpb::ProblemView made_problem(const qpb_problem* problem) {
  const qpb::ProblemView v = view(problem);
  qpb::dims_of(v);
  if (!v.amplitude || !v.support) {
    throw qpb::InvalidArgument("problem arrays do not match its shape; build it with make_problem");
  }
  return v;
}

}  // namespace

qpb_status qpb_create(const qpb_problem* problem, const qpb_options* options, qpb_solver** out) {
  return guarded([&] {
    require(out != nullptr, "out is NULL");
    *out = nullptr;
    const qpb::SolverOptions o = options_of(options);
    const qpb::ProblemView v = made_problem(problem);
    if (!qpb_cuda_available()) throw std::runtime_error("no CUDA device available");
    qpb::trace("qpb_create: starts=%d batch=%d variant=%d shape=%lld,%lld,%lld", o.starts, o.batch,
               options->variant, v.shape[0], v.shape[1], v.shape[2]);
    *out = new qpb_solver({v}, o);
    qpb::trace("qpb_create: solver %p ready", static_cast<void*>(*out));
  });
}

qpb_status qpb_create_device(const qpb_problem* problem, const qpb_options* options,
                             qpb_solver** out) {
  return guarded([&] {
    require(out != nullptr, "out is NULL");
    *out = nullptr;
    const qpb::SolverOptions o = options_of(options);
    qpb::ProblemView v = made_problem(problem);
    v.on_device = true;
    require_aligned(v.amplitude, alignof(float), "amplitude");
    require_aligned(o.start, alignof(float2), "options->start");
    if (!qpb_cuda_available()) throw std::runtime_error("no CUDA device available");
    *out = new qpb_solver({v}, o);
  });
}

qpb_status qpb_reset(qpb_solver* solver, const qpb_problem* problems, size_t n_problems,
                     uint64_t seed, const float* start) {
  return guarded([&] {
    require(solver != nullptr, "solver is NULL");
    require(problems != nullptr && n_problems > 0, "no problems");
    std::vector<qpb::ProblemView> views;
    for (size_t q = 0; q < n_problems; ++q) views.push_back(made_problem(problems + q));
    use_solver_device(solver);
    solver->impl.reset(views, seed, reinterpret_cast<const float2*>(start));
  });
}

qpb_status qpb_results_device(qpb_solver* solver, float* objects, uint8_t* supports,
                              float* errors) {
  return guarded([&] {
    require(solver != nullptr, "solver is NULL");
    require_aligned(objects, alignof(float2), "objects");
    use_solver_device(solver);
    solver->impl.results_device(reinterpret_cast<float2*>(objects), supports, errors);
  });
}

qpb_status qpb_make_problem_device(const float* intensity, int ndim, const int64_t* shape,
                                   const uint8_t* support, const uint8_t* mask,
                                   float support_threshold, float* amplitude_out,
                                   uint8_t* mask_out, uint8_t* support_out, void* stream) {
  return guarded([&] {
    numel_checked(ndim, shape);
    require(intensity && amplitude_out && mask_out && support_out, "NULL array");
    long long sh[3] = {0, 0, 0};
    for (int k = 0; k < ndim; ++k) sh[k] = shape[k];
    qpb::make_problem_device(intensity, ndim, sh, support, mask, support_threshold, amplitude_out,
                             mask_out, support_out, static_cast<cudaStream_t>(stream));
  });
}

qpb_status qpb_create_batch(const qpb_problem* problems, size_t n_problems,
                            const qpb_options* options, qpb_solver** out) {
  return guarded([&] {
    require(out != nullptr, "out is NULL");
    *out = nullptr;
    require(problems != nullptr && n_problems > 0, "no problems");
    const qpb::SolverOptions o = options_of(options);
    std::vector<qpb::ProblemView> views;
    for (size_t q = 0; q < n_problems; ++q) views.push_back(made_problem(problems + q));
    if (!qpb_cuda_available()) throw std::runtime_error("no CUDA device available");
    *out = new qpb_solver(views, o);
  });
}

qpb_status qpb_run(qpb_solver* solver, const qpb_op* ops, size_t n_ops) {
  return guarded([&] {
    require(solver != nullptr, "solver is NULL");
    require(ops != nullptr || n_ops == 0, "ops is NULL");
    static_assert(sizeof(qpb_op) == sizeof(qpb::OpDesc));
    if (qpb::tracing()) {
      qpb::trace("qpb_run solver=%p ops=%p n_ops=%zu", static_cast<void*>(solver),
                 static_cast<const void*>(ops), n_ops);
      for (size_t i = 0; i < n_ops; ++i) {
        qpb::trace("  op[%zu] kind=%d n=%d beta=%g thr=%g sigma=%g method=%d axis=%d", i,
                   ops[i].kind, ops[i].n, ops[i].beta, ops[i].threshold, ops[i].sigma,
                   ops[i].method, ops[i].axis);
      }
    }
    qpb::validate_recipe(reinterpret_cast<const qpb::OpDesc*>(ops), n_ops);
    qpb::trace("qpb_run: recipe valid, selecting device %d", solver->impl.device());
    use_solver_device(solver);
    solver->impl.run(reinterpret_cast<const qpb::OpDesc*>(ops), n_ops);
  });
}

uint64_t qpb_kernel_launches(void) { return qpb::launches(); }

qpb_status qpb_tuning_report(char* out, size_t len) {
  return guarded([&] {
    require(out != nullptr && len > 0, "NULL argument");
    const std::string report = qpb::tuning_report();
    std::strncpy(out, report.c_str(), len - 1);
    out[len - 1] = '\0';
  });
}

qpb_status qpb_profile_passes(qpb_solver* solver, int iterations, double* ms_out, int* n_passes) {
  return guarded([&] {
    require(solver && ms_out && n_passes, "NULL argument");
    use_solver_device(solver);
    *n_passes = solver->impl.profile_passes(iterations, ms_out);
  });
}

qpb_status qpb_set_wait_limit(qpb_solver* solver, int polls, int starve) {
  return guarded([&] {
    require(solver != nullptr, "solver is NULL");
    require(polls >= 1, "polls must be >= 1");
    use_solver_device(solver);
    solver->impl.set_wait(polls, starve != 0);
  });
}

qpb_status qpb_set_progress(qpb_solver* solver, qpb_progress_fn fn, void* user) {
  return guarded([&] {
    require(solver != nullptr, "solver is NULL");
    solver->impl.set_progress(fn, user);
  });
}

qpb_status qpb_error_count(const qpb_solver* solver, size_t* count) {
  return guarded([&] {
    require(solver && count, "NULL argument");
    *count = solver->impl.error_count();
  });
}

qpb_status qpb_starts(const qpb_solver* solver, int* starts) {
  return guarded([&] {
    require(solver && starts, "NULL argument");
    *starts = solver->impl.starts();
  });
}

qpb_status qpb_results(qpb_solver* solver, float* objects, uint8_t* supports, float* errors) {
  return guarded([&] {
    require(solver != nullptr, "solver is NULL");
    use_solver_device(solver);
    solver->impl.results(reinterpret_cast<float2*>(objects), supports, errors);
  });
}

void qpb_destroy(qpb_solver* solver) {
  if (!solver) return;
  cudaSetDevice(solver->impl.device());
  delete solver;
}

qpb_status qpb_aligned_error(const float* a, const float* reference, int ndim,
                             const int64_t* shape, int batch, float* out) {
  return guarded([&] {
    require(a && reference && out, "NULL array");
    numel_checked(ndim, shape);
    require(batch >= 1, "batch must be >= 1");
    long long sh[3] = {0, 0, 0};
    for (int k = 0; k < ndim; ++k) sh[k] = shape[k];
    qpb::aligned_error(reinterpret_cast<const float2*>(a), reinterpret_cast<const float2*>(reference),
                       ndim, sh, batch, out);
  });
}

qpb_status qpb_align(const float* a, const float* reference, int ndim, const int64_t* shape,
                     int batch, float* errors, float* aligned, float* mean) {
  return guarded([&] {
    require(a && reference, "NULL array");
    numel_checked(ndim, shape);
    require(batch >= 1, "batch must be >= 1");
    long long sh[3] = {0, 0, 0};
    for (int k = 0; k < ndim; ++k) sh[k] = shape[k];
    qpb::align(reinterpret_cast<const float2*>(a), reinterpret_cast<const float2*>(reference), ndim,
               sh, batch, errors, reinterpret_cast<float2*>(aligned),
               reinterpret_cast<float2*>(mean));
  });
}

qpb_status qpb_simulate_intensity(const float* object, int ndim, const int64_t* shape,
                                  float* out) {
  return guarded([&] {
    require(object && out, "NULL array");
    numel_checked(ndim, shape);
    long long sh[3] = {0, 0, 0};
    for (int k = 0; k < ndim; ++k) sh[k] = shape[k];
    qpb::simulate_intensity(reinterpret_cast<const float2*>(object), ndim, sh, out);
  });
}

qpb_status qpb_modulus_project(const qpb_problem* problem, float* obj, int amp_storage,
                               float* error_out) {
  return guarded([&] {
    require(obj != nullptr, "obj is NULL");
    if (!qpb_cuda_available()) throw std::runtime_error("no CUDA device available");
    const float e = qpb::modulus_project(view(problem), reinterpret_cast<float2*>(obj),
                                         storage_of(amp_storage));
    if (error_out) *error_out = e;
  });
}

qpb_status qpb_support_project(const uint8_t* support, float* obj, size_t count) {
  return guarded([&] {
    require(support && obj, "NULL array");
    qpb::support_project_host(support, reinterpret_cast<float2*>(obj),
                              static_cast<long long>(count));
  });
}

qpb_status qpb_gaussian_blur(const float* image, int ndim, const int64_t* shape, float sigma,
                             float* out) {
  return guarded([&] {
    numel_checked(ndim, shape);
    require(image && out, "NULL array");
    long long sh[3] = {0, 0, 0};
    for (int a = 0; a < ndim; ++a) sh[a] = shape[a];
    qpb::gaussian_blur(image, ndim, sh, sigma, out);
  });
}

}  // extern "C"
