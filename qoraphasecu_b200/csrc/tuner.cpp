// Autotuner for the batched schedule: how many starts share one launch.
//
// Starts are independent, so any grouping gives the same iterates; what
// changes is how the work fills the GPU. One group of all starts is a single
// chain of kernels per iteration whose last CTAs run with the SMs half idle;
// several smaller groups become parallel branches of the captured graph, and
// one group's modulus pass then overlaps another's update pass. The best
// split depends on the shape, the start count and the device, so it is
// measured: each candidate runs a short RAAR stage on a scratch solver built
// from the same problem, and the fastest is cached for the process.

#include <chrono>
#include <cstdlib>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>
#include <vector>

#include "solver.hpp"

namespace qpb {

namespace {

using Key = std::tuple<int, int, int, int, int, int>;  // device, d0, d1, d2, starts, storage

std::mutex g_mutex;
std::map<Key, int> g_choice;
std::map<Key, std::vector<std::pair<int, double>>> g_timings;

bool tuning_enabled() {
  const char* v = std::getenv("QPB_TUNE");
  return !(v && *v == '0');
}

double time_candidate(const ProblemView& problem, const SolverOptions& base, int batch) {
  SolverOptions o = base;
  o.batch = batch;
  o.tune = false;
  o.start = nullptr;
  o.seed = 0;
  o.stream = nullptr;
  o.sync_every = 10;
  o.variant = Variant::kBatched;
  Solver solver(problem, o);
  const OpDesc raar{kOpRAAR, 10, 0.9f, 0.0f, 0.0f, 0, 0};
  solver.run(&raar, 1);  // captures the graph
  double best = 1e30;
  for (int rep = 0; rep < 2; ++rep) {
    const auto t0 = std::chrono::steady_clock::now();
    solver.run(&raar, 1);
    const auto t1 = std::chrono::steady_clock::now();
    best = std::min(best, std::chrono::duration<double>(t1 - t0).count());
  }
  return best;
}

}  // namespace

int tuned_batch(const ProblemView& problem, const SolverOptions& options) {
  const int starts = options.starts;
  if (starts < 2 || !tuning_enabled()) return starts;
  const Dims3 d = dims_of(problem);
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  const Key key{device, d.d0, d.d1, d.d2, starts, static_cast<int>(options.amp_storage)};
  std::lock_guard<std::mutex> lock(g_mutex);
  if (auto it = g_choice.find(key); it != g_choice.end()) return it->second;
  std::vector<int> candidates;
  for (int parts : {1, 2, 4, 8}) {
    if (starts % parts == 0 && (parts == 1 || starts / parts >= 1)) candidates.push_back(starts / parts);
  }
  int best = starts;
  double best_time = 1e30;
  std::vector<std::pair<int, double>> timings;
  for (int batch : candidates) {
    const double t = time_candidate(problem, options, batch);
    timings.emplace_back(batch, t);
    if (t < best_time * 0.98) {  // prefer fewer groups unless clearly faster
      best_time = t;
      best = batch;
    }
  }
  g_choice[key] = best;
  g_timings[key] = timings;
  trace("tuned batch for %dx%dx%d, %d starts: %d", d.d0, d.d1, d.d2, starts, best);
  return best;
}

std::string tuning_report() {
  std::lock_guard<std::mutex> lock(g_mutex);
  std::ostringstream out;
  for (const auto& [key, choice] : g_choice) {
    const auto& [device, d0, d1, d2, starts, storage] = key;
    out << "device " << device << " shape " << d0 << "x" << d1 << "x" << d2 << " starts "
        << starts << " storage " << storage << ": batch " << choice << " (";
    bool first = true;
    for (const auto& [batch, t] : g_timings[key]) {
      out << (first ? "" : ", ") << batch << ": " << t * 1e3 << " ms";
      first = false;
    }
    out << ")\n";
  }
  return out.str();
}

}  // namespace qpb
