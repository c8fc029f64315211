// Many problems of uneven shapes reconstructed together.
//
// Problems are grouped into shape classes (first-appearance order); each class
// is one Solver over all its problems (one batched launch per pass or resident
// chunk for all of them, its schedule picked by the autotuner for that shape
// and start count). Every chunk of iterations of every class is captured into
// ONE graph per chunk length: the classes are parallel branches of it, so the
// small problems fill the SMs the large ones leave idle. Shrinkwrap and detwin
// run between chunks, as in a single solver. A batch of one problem is exactly
// a Solver.
#pragma once

#include <map>
#include <memory>
#include <vector>

#include "solver.hpp"

namespace qpb {

class BatchSolver {
 public:
  // options.starts = starts per problem; options.start, when given, holds every
  // problem's starts in problem order (starts * numel(q) complex64 each).
  BatchSolver(const std::vector<ProblemView>& problems, const SolverOptions& options);
  ~BatchSolver();
  BatchSolver(const BatchSolver&) = delete;
  BatchSolver& operator=(const BatchSolver&) = delete;

  void run(const OpDesc* ops, std::size_t count);
  // Solver::reset for every shape class: new problems (the same count, problem
  // q of problem q's shape at construction, host or device arrays as then),
  // new starts drawn from `seed` as a new batch would draw them, or given.
  void reset(std::vector<ProblemView> problems, std::uint64_t seed, const float2* start);
  bool on_device() const { return on_device_; }
  std::size_t error_count() const { return classes_[0].solver->error_count(); }
  int starts() const { return spp_ * static_cast<int>(where_.size()); }
  int problems() const { return static_cast<int>(where_.size()); }
  int classes() const { return static_cast<int>(classes_.size()); }
  int device() const { return select_.device; }
  // Problem order; problem q's block holds starts * numel(q) objects/supports
  // and starts * error_count() errors, blocks back to back.
  void results(float2* objects, std::uint8_t* supports, float* errors);
  // Objects and supports into device memory (one shape only); errors on the host.
  void results_device(float2* objects, std::uint8_t* supports, float* errors);
  void set_progress(ProgressFn fn, void* user);
  // One shape class only (the per-pass profile of its solver).
  int profile_passes(int iterations, double* ms);
  // Solver::set_wait for every shape class; the batch's own captured graphs
  // are dropped too.
  void set_wait(int tries, bool starve);

 private:
  struct Class {
    std::vector<int> members;  // problem indices, in order
    std::unique_ptr<Solver> solver;
  };
  void report(int iteration);

  DeviceSelect select_;
  Stream stream_;
  int spp_;
  int every_;
  bool batched_;  // chunks captured into graphs (else launched directly)
  bool on_device_;  // problem arrays given as device pointers
  std::vector<Class> classes_;
  std::vector<std::pair<int, int>> where_;  // problem -> (class, index in class)
  std::vector<long long> numel_;            // per problem
  std::vector<std::unique_ptr<Stream>> branches_;  // one per class
  std::vector<cudaEvent_t> events_;                // fork + one join per class
  std::map<int, std::unique_ptr<Graph>> graphs_;   // by chunk length
  ProgressFn progress_ = nullptr;
  void* progress_user_ = nullptr;
  int iteration_ = 0;
};

}  // namespace qpb
