// qpcu::Solver over libqpb.so: the adapter that makes the B200 backend a
// QoraPhaseCU backend.
//
// Compiled inside the reference project, against its public headers
// (include/qoraphasecu/solver.hpp:40-74, recipe.hpp:8-86, problem.hpp:20-47)
// and src/core/backends.hpp:9-10. It converts the reference's types at the C
// ABI of include/qpb.h and nothing else: Problem -> qpb_problem, Options ->
// qpb_options, each recipe Op -> qpb_op (the seven fields of the reference's
// Python op tuple, python/bindings.cpp:22-23), qpb_results -> Reconstruction,
// qpb_status -> the reference's exception types (std::invalid_argument for
// bad inputs, src/core/solver.cpp:62-78; std::runtime_error for device
// failures, src/cuda/common.cuh:15-31). Options::variant is ignored, as the
// reference's CPU backend ignores it.
//
// A maintainer adds `Backend::b200` to the enum (solver.hpp:16), its name to
// to_string/parse_backend (solver.cpp:13-48) and one case to make_solver's
// switch (solver.cpp:79-85) that returns detail::make_b200_solver.

#include <complex>
#include <cstdint>
#include <memory>
#include <span>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <variant>
#include <vector>

#include "qoraphasecu/qoraphasecu.hpp"
#include "qpb.h"

namespace qpcu::detail {

std::unique_ptr<Solver> make_b200_solver(const Problem& problem, const Options& options);

namespace {

void check(qpb_status status) {
  if (status == QPB_OK) return;
  if (status == QPB_INVALID_ARGUMENT) throw std::invalid_argument(qpb_last_error());
  throw std::runtime_error(qpb_last_error());
}

qpb_op to_op(const Op& op) {
  qpb_op o{};
  std::visit(
      [&](const auto& s) {
        using T = std::decay_t<decltype(s)>;
        if constexpr (std::is_same_v<T, ER>) {
          o.kind = QPB_OP_ER;
          o.n = s.n;
        } else if constexpr (std::is_same_v<T, HIO>) {
          o.kind = QPB_OP_HIO;
          o.n = s.n;
          o.beta = s.beta;
        } else if constexpr (std::is_same_v<T, RAAR>) {
          o.kind = QPB_OP_RAAR;
          o.n = s.n;
          o.beta = s.beta;
        } else if constexpr (std::is_same_v<T, Shrinkwrap>) {
          o.kind = QPB_OP_SHRINKWRAP;
          o.threshold = s.threshold;
          o.sigma = s.sigma;
          o.method = s.method == Threshold::rms ? 1 : 0;
        } else if constexpr (std::is_same_v<T, DetwinBegin>) {
          o.kind = QPB_OP_DETWIN_BEGIN;
          o.axis = s.axis;
        } else {
          o.kind = QPB_OP_DETWIN_END;
        }
      },
      op);
  return o;
}

class B200Solver final : public Solver {
 public:
  B200Solver(const Problem& p, const Options& o) : shape_(p.shape), progress_(o.progress) {
    qpb_problem prob{};
    prob.ndim = static_cast<int>(p.shape.size());
    for (std::size_t a = 0; a < p.shape.size() && a < 3; ++a) {
      prob.shape[a] = static_cast<int64_t>(p.shape[a]);
    }
    prob.amplitude = p.amplitude.data();
    prob.mask = p.mask.data();
    prob.support = p.support.data();
    qpb_options opts{};
    opts.starts = o.starts;
    opts.batch = o.batch;
    opts.seed = o.seed;
    opts.start = o.start.empty() ? nullptr : reinterpret_cast<const float*>(o.start.data());
    opts.sync_every = o.sync_every;
    opts.variant = QPB_VARIANT_BATCHED;
    opts.amp_storage = QPB_AMP_F32;
    opts.device = -1;
    opts.stream = nullptr;
    opts.schedule = QPB_SCHEDULE_AUTO;
    check(qpb_create(&prob, &opts, &solver_));
    if (progress_) {
      check(qpb_set_progress(
          solver_,
          [](void* self, int iteration, const float* errors, int count) {
            static_cast<B200Solver*>(self)->progress_(
                iteration, std::span<const float>(errors, static_cast<std::size_t>(count)));
          },
          this));
    }
  }
  B200Solver(const B200Solver&) = delete;
  B200Solver& operator=(const B200Solver&) = delete;
  ~B200Solver() override { qpb_destroy(solver_); }

  void run(const Recipe& recipe) override {
    std::vector<qpb_op> ops;
    ops.reserve(recipe.ops.size());
    for (const Op& op : recipe.ops) ops.push_back(to_op(op));
    check(qpb_run(solver_, ops.data(), ops.size()));
  }

  std::vector<Reconstruction> results() const override {
    int starts = 0;
    std::size_t count = 0;
    check(qpb_starts(solver_, &starts));
    check(qpb_error_count(solver_, &count));
    const std::size_t n = numel(shape_);
    std::vector<Complex> objects(n * static_cast<std::size_t>(starts));
    std::vector<std::uint8_t> supports(n * static_cast<std::size_t>(starts));
    std::vector<float> errors(count * static_cast<std::size_t>(starts));
    check(qpb_results(solver_, reinterpret_cast<float*>(objects.data()), supports.data(),
                      errors.data()));
    std::vector<Reconstruction> out;
    out.reserve(static_cast<std::size_t>(starts));
    for (std::size_t s = 0; s < static_cast<std::size_t>(starts); ++s) {
      Reconstruction r;
      r.object.assign(objects.begin() + s * n, objects.begin() + (s + 1) * n);
      r.support.assign(supports.begin() + s * n, supports.begin() + (s + 1) * n);
      r.errors.assign(errors.begin() + s * count, errors.begin() + (s + 1) * count);
      out.push_back(std::move(r));
    }
    return out;
  }

 private:
  Shape shape_;
  Progress progress_;
  qpb_solver* solver_ = nullptr;
};

}  // namespace

std::unique_ptr<Solver> make_b200_solver(const Problem& problem, const Options& options) {
  if (!qpb_cuda_available()) throw std::runtime_error("no CUDA device available");
  return std::make_unique<B200Solver>(problem, options);
}

}  // namespace qpcu::detail
