// Many problems of uneven shapes in one graph per chunk of iterations.

#include "batch.hpp"

#include <algorithm>
#include <array>
#include <cstring>
#include <stdexcept>
#include <string>

#include "nvtx_range.hpp"

namespace qpb {

BatchSolver::BatchSolver(const std::vector<ProblemView>& problems, const SolverOptions& options)
    : select_(options.device),
      stream_(options.stream),
      spp_(options.starts),
      every_(options.sync_every),
      batched_(options.variant != Variant::kPlain),
      on_device_(!problems.empty() && problems[0].on_device) {
  if (problems.empty()) throw InvalidArgument("no problems");
  if (options.starts < 1) throw InvalidArgument("starts must be >= 1");
  if (options.sync_every < 1) throw InvalidArgument("sync_every must be >= 1");
  std::vector<std::array<long long, 4>> keys;
  where_.resize(problems.size());
  numel_.resize(problems.size());
  for (std::size_t q = 0; q < problems.size(); ++q) {
    const Dims3 d = dims_of(problems[q]);
    numel_[q] = d.n();
    const std::array<long long, 4> key{problems[q].ndim, d.d0, d.d1, d.d2};
    auto it = std::find(keys.begin(), keys.end(), key);
    if (it == keys.end()) {
      keys.push_back(key);
      classes_.emplace_back();
      it = keys.end() - 1;
    }
    const int c = static_cast<int>(it - keys.begin());
    where_[q] = {c, static_cast<int>(classes_[c].members.size())};
    classes_[c].members.push_back(static_cast<int>(q));
  }
  if (options.start && problems[0].on_device && classes_.size() > 1) {
    throw InvalidArgument("given starts on the device need problems of one shape");
  }
  std::vector<long long> start_off(problems.size(), 0);
  for (std::size_t q = 1; q < problems.size(); ++q) {
    start_off[q] = start_off[q - 1] + static_cast<long long>(spp_) * numel_[q - 1];
  }
  for (Class& c : classes_) {
    std::vector<ProblemView> views;
    for (int q : c.members) views.push_back(problems[q]);
    SolverOptions o = options;
    o.stream = stream_;
    o.device = select_.device;
    std::vector<float2> given;
    if (options.start && classes_.size() > 1) {
      for (int q : c.members) {
        const float2* src = options.start + start_off[q];
        given.insert(given.end(), src, src + static_cast<std::size_t>(spp_) * numel_[q]);
      }
      o.start = given.data();
    }
    c.solver = std::make_unique<Solver>(views, o);
  }
  if (classes_.size() > 1) {
    for (std::size_t c = 0; c < classes_.size(); ++c) branches_.push_back(std::make_unique<Stream>());
    events_.resize(classes_.size() + 1);
    for (auto& e : events_) QPB_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  trace("batch: %zu problems in %zu shape classes", problems.size(), classes_.size());
}

BatchSolver::~BatchSolver() {
  cudaSetDevice(select_.device);
  cudaStreamSynchronize(stream_);
  graphs_.clear();
  for (cudaEvent_t e : events_) cudaEventDestroy(e);
}

void BatchSolver::set_progress(ProgressFn fn, void* user) {
  if (classes_.size() == 1) {
    classes_[0].solver->set_progress(fn, user);
    return;
  }
  progress_ = fn;
  progress_user_ = user;
}

void BatchSolver::report(int iteration) {
  std::vector<float> all(static_cast<std::size_t>(starts()));
  for (const Class& c : classes_) {
    const std::vector<float> latest = c.solver->latest_errors();
    for (std::size_t j = 0; j < c.members.size(); ++j) {
      std::copy_n(latest.begin() + static_cast<long long>(j) * spp_, spp_,
                  all.begin() + static_cast<long long>(c.members[j]) * spp_);
    }
  }
  progress_(progress_user_, iteration, all.data(), starts());
}

void BatchSolver::run(const OpDesc* ops, std::size_t count) {
  if (classes_.size() == 1) {
    classes_[0].solver->run(ops, count);
    return;
  }
  validate_recipe(ops, count);
  const NvtxRange recipe_range("batch recipe", recipe_iterations(ops, count));
  for (Class& c : classes_) c.solver->begin_run(ops, count);
  for (std::size_t i = 0; i < count; ++i) {
    const OpDesc& o = ops[i];
    const NvtxRange stage_range(op_name(o.kind), o.n);
    Coefficients co{};
    switch (o.kind) {
      case kOpER:
        co = er_coefficients();
        break;
      case kOpHIO:
        co = hio_coefficients(o.beta);
        break;
      case kOpRAAR:
        co = raar_coefficients(o.beta);
        break;
      default:
        for (Class& c : classes_) c.solver->apply(o);
        continue;
    }
    for (Class& c : classes_) c.solver->begin_iterate(co);
    for (int done = 0; done < o.n;) {
      const int len = classes_[0].solver->chunk_length(o.n - done);
      if (batched_) {
        // graphs by chunk length and wave storage (the mixed variant switches it)
        const int key = 2 * len + (classes_[0].solver->wave_half() ? 1 : 0);
        auto it = graphs_.find(key);
        if (it == graphs_.end()) {
          for (Class& c : classes_) c.solver->prepare_branches();
          const unsigned long long before = launches();
          QPB_CHECK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
          try {
            QPB_CHECK(cudaEventRecord(events_[0], stream_));
            for (std::size_t k = 0; k < classes_.size(); ++k) {
              cudaStream_t b = *branches_[k];
              QPB_CHECK(cudaStreamWaitEvent(b, events_[0], 0));
              classes_[k].solver->enqueue_chunk_body(len, b);
              QPB_CHECK(cudaEventRecord(events_[k + 1], b));
              QPB_CHECK(cudaStreamWaitEvent(stream_, events_[k + 1], 0));
            }
          } catch (...) {
            cudaGraph_t broken{};
            cudaStreamEndCapture(stream_, &broken);
            if (broken) cudaGraphDestroy(broken);
            throw;
          }
          cudaGraph_t graph{};
          QPB_CHECK(cudaStreamEndCapture(stream_, &graph));
          const unsigned long long kernels = launches() - before;
          count_launches(0ULL - kernels);  // counted again on every replay
          it = graphs_.emplace(key, std::make_unique<Graph>(graph, kernels)).first;
        }
        it->second->launch(stream_);
      } else {
        for (Class& c : classes_) c.solver->enqueue_chunk_body(len, stream_);
      }
      for (Class& c : classes_) c.solver->end_chunk(len);
      iteration_ += len;
      done += len;
      if (progress_ && iteration_ % every_ == 0) report(iteration_);
    }
  }
  for (Class& c : classes_) c.solver->end_run();
}

void BatchSolver::set_wait(int tries, bool starve) {
  stream_.sync();
  graphs_.clear();
  for (Class& c : classes_) c.solver->set_wait(tries, starve);
}

void BatchSolver::results(float2* objects, std::uint8_t* supports, float* errors) {
  if (classes_.size() == 1) {
    classes_[0].solver->results(objects, supports, errors);
    return;
  }
  const std::size_t errs = error_count();
  std::vector<long long> off(where_.size(), 0);
  for (std::size_t q = 1; q < where_.size(); ++q) off[q] = off[q - 1] + spp_ * numel_[q - 1];
  for (Class& c : classes_) {
    // each member problem's block goes straight to its place in the output
    std::vector<float2*> o(c.members.size(), nullptr);
    std::vector<std::uint8_t*> s(c.members.size(), nullptr);
    std::vector<float*> e(c.members.size(), nullptr);
    for (std::size_t j = 0; j < c.members.size(); ++j) {
      const int q = c.members[j];
      if (objects) o[j] = objects + off[q];
      if (supports) s[j] = supports + off[q];
      if (errors) e[j] = errors + static_cast<std::size_t>(q) * spp_ * errs;
    }
    c.solver->results_per_problem(objects ? o.data() : nullptr, supports ? s.data() : nullptr,
                                  errors ? e.data() : nullptr);
  }
}

void BatchSolver::reset(std::vector<ProblemView> problems, std::uint64_t seed,
                        const float2* start) {
  if (problems.size() != where_.size()) {
    throw InvalidArgument("reset needs as many problems as the batch was built with");
  }
  for (std::size_t q = 0; q < problems.size(); ++q) {
    problems[q].on_device = on_device_;
    if (dims_of(problems[q]).n() != numel_[q]) {
      throw InvalidArgument("reset needs problem " + std::to_string(q) + " in its original shape");
    }
  }
  if (classes_.size() == 1) {
    classes_[0].solver->reset(problems, seed, start);
    iteration_ = 0;
    return;
  }
  if (start && on_device_) throw InvalidArgument("given starts on the device need problems of one shape");
  std::vector<long long> start_off(problems.size(), 0);
  for (std::size_t q = 1; q < problems.size(); ++q) {
    start_off[q] = start_off[q - 1] + static_cast<long long>(spp_) * numel_[q - 1];
  }
  for (Class& c : classes_) {
    std::vector<ProblemView> views;
    std::vector<float2> given;
    for (int q : c.members) {
      views.push_back(problems[q]);
      if (start) {
        const float2* src = start + start_off[q];
        given.insert(given.end(), src, src + static_cast<std::size_t>(spp_) * numel_[q]);
      }
    }
    c.solver->reset(views, seed, start ? given.data() : nullptr);
  }
  iteration_ = 0;
}

void BatchSolver::results_device(float2* objects, std::uint8_t* supports, float* errors) {
  if (classes_.size() != 1) throw InvalidArgument("device results need problems of one shape");
  classes_[0].solver->results_device(objects, supports, errors);
}

int BatchSolver::profile_passes(int iterations, double* ms) {
  if (classes_.size() != 1) {
    throw InvalidArgument("profile_passes needs problems of one shape");
  }
  return classes_[0].solver->profile_passes(iterations, ms);
}

}  // namespace qpb
