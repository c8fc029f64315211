// Autotuner for the batched schedule: the resident kernel, or streamed passes
// with how many starts per launch.
//
// Starts are independent, so any schedule gives the same iterates; what
// changes is how the work fills the GPU. The resident kernel keeps each start
// in a cluster's shared memory for a whole chunk of iterations, but one start
// takes up to 8 SMs, so few starts leave SMs idle. With streamed passes, one
// group of all starts is a single chain of kernels per iteration whose last
// CTAs run with the SMs half idle; several smaller groups become parallel
// branches of the captured graph, and one group's modulus pass then overlaps
// another's update pass. The best choice depends on the shape, the start count
// and the device, so it is measured: each candidate runs a short RAAR stage
// (two chunks of the caller's length) on a scratch solver built from the same
// problem, and the fastest is cached for the process.

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "persistent.cuh"
#include "resident.cuh"
#include "solver.hpp"

namespace qpb {

namespace {

// device, d0, d1, d2, starts, amplitude storage, resident kernel among the
// candidates, variant (fp16 storage changes the passes' cost)
using Key = std::tuple<int, int, int, int, int, int, bool, int>;

std::mutex g_mutex;
std::map<Key, TunedSchedule> g_choice;
// Timings per candidate: batch (starts per launch) or 0 for the resident kernel.
std::map<Key, std::vector<std::pair<int, double>>> g_timings;

bool tuning_enabled() {
  const char* v = std::getenv("QPB_TUNE");
  return !(v && *v == '0');
}

// batch > 0: streamed passes with that many starts per launch; 0: the
// resident kernel; kPersistentCandidate: the persistent kernel.
constexpr int kPersistentCandidate = -1;

double time_candidate(const ProblemView& problem, const SolverOptions& base, int batch) {
  SolverOptions o = base;
  o.batch = batch > 0 ? batch : 0;
  o.schedule = batch == 0                      ? Schedule::kResident
               : batch == kPersistentCandidate ? Schedule::kPersistent
                                               : Schedule::kStreamed;
  o.tune = false;
  o.start = nullptr;
  o.seed = 0;
  o.stream = nullptr;
  // The caller's chunk length (10..100 iterations), so that each candidate
  // replays the graphs the caller's run would replay; two chunks per timing
  // keep the host's share of the wall time small.
  o.sync_every = std::max(10, std::min(base.sync_every, 100));
  o.variant = base.variant == Variant::kPlain ? Variant::kBatched : base.variant;
  Solver solver(problem, o);
  const OpDesc raar{kOpRAAR, 2 * o.sync_every, 0.9f, 0.0f, 0.0f, 0, 0};
  solver.run(&raar, 1);  // captures the graph
  double best = 1e30;
  for (int rep = 0; rep < 3; ++rep) {
    const auto t0 = std::chrono::steady_clock::now();
    solver.run(&raar, 1);
    const auto t1 = std::chrono::steady_clock::now();
    best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
  }
  return best;
}

}  // namespace

TunedSchedule tuned_schedule(const ProblemView& problem, const SolverOptions& options) {
  const int starts = options.starts;
  const bool resident_ok = options.schedule != Schedule::kStreamed;
  if (!tuning_enabled() || (starts < 2 && !resident_ok)) return {starts, false};
  const Dims3 d = dims_of(problem);
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  const Key key{device, d.d0, d.d1, d.d2, starts, static_cast<int>(options.amp_storage),
                resident_ok, static_cast<int>(options.variant)};
  std::lock_guard<std::mutex> lock(g_mutex);
  if (auto it = g_choice.find(key); it != g_choice.end()) return it->second;
  std::vector<int> candidates;
  const bool resident_here = resident_ok && resident_supports(problem.ndim, d.d1, d.d2) &&
                             options.variant == Variant::kBatched;
  const bool persistent_here = options.schedule != Schedule::kStreamed &&
                               options.variant == Variant::kBatched &&
                               persistent_supports(problem.ndim, d.d1, d.d2);
  if (resident_here) candidates.push_back(0);
  if (persistent_here) candidates.push_back(kPersistentCandidate);
  for (int parts : {1, 2, 4, 8, 16}) {
    if (starts % parts == 0 && starts / parts >= 1) candidates.push_back(starts / parts);
  }
  TunedSchedule best{starts, false};
  double best_time = 1e30;
  std::vector<std::pair<int, double>> timings;
  for (int batch : candidates) {
    double t = 0.0;
    try {
      t = time_candidate(problem, options, batch);
    } catch (const Timeout&) {
      throw;
    } catch (const std::exception& e) {
      // a candidate this device cannot run is left out
      trace("tuner: candidate %d failed: %s", batch, e.what());
      continue;
    }
    timings.emplace_back(batch, t);
    if (t < best_time * 0.98) {  // prefer earlier candidates unless clearly slower
      best_time = t;
      best = batch == 0                      ? TunedSchedule{starts, true, false}
             : batch == kPersistentCandidate ? TunedSchedule{starts, false, true}
                                             : TunedSchedule{batch, false, false};
    }
  }
  g_choice[key] = best;
  g_timings[key] = timings;
  trace("tuned schedule for %dx%dx%d, %d starts: %s batch %d", d.d0, d.d1, d.d2, starts,
        best.resident ? "resident" : (best.persistent ? "persistent" : "streamed"), best.batch);
  return best;
}

std::string tuning_report() {
  std::lock_guard<std::mutex> lock(g_mutex);
  std::ostringstream out;
  for (const auto& [key, choice] : g_choice) {
    const auto& [device, d0, d1, d2, starts, storage, resident_ok, variant] = key;
    out << "device " << device << " shape " << d0 << "x" << d1 << "x" << d2 << " starts "
        << starts << " storage " << storage
        << (variant == static_cast<int>(Variant::kHalf)    ? " half"
            : variant == static_cast<int>(Variant::kMixed) ? " mixed"
                                                           : "")
        << ": "
        << (choice.resident     ? std::string("resident")
            : choice.persistent ? std::string("persistent")
                                : "batch " + std::to_string(choice.batch))
        << " (";
    bool first = true;
    for (const auto& [batch, t] : g_timings[key]) {
      if (batch == 0) {
        out << (first ? "" : ", ") << "resident (" << resident_max_clusters(d2) << " clusters of "
            << resident_cluster(d2) << " CTAs at once): " << t * 1e3 << " ms";
      } else if (batch == kPersistentCandidate) {
        out << (first ? "" : ", ") << "persistent (" << persistent_grid(d1, d2)
            << " CTAs): " << t * 1e3 << " ms";
      } else {
        out << (first ? "" : ", ") << batch << ": " << t * 1e3 << " ms";
      }
      first = false;
    }
    out << ")\n";
  }
  return out.str();
}

}  // namespace qpb
