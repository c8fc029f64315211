// The B200 reconstruction solver: every start's iterate resident in HBM in FFT
// order, iterations as fused line passes, batched starts captured in CUDA
// graphs. It implements the contract of QoraPhaseCU's qpcu::Solver
// (include/qoraphasecu/solver.hpp:67-74): construction draws the starts, run()
// continues from the current state and appends one error per iteration,
// results() returns centre-origin objects, supports and error histories.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "aux_kernels.cuh"
#include "common.cuh"
#include "fft_plan.hpp"
#include "line_pass.cuh"

namespace qpb {

// Owning device allocation.
template <class T>
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(std::size_t count) : count_(count) {
    if (!count) return;
    const cudaError_t status = cudaMalloc(reinterpret_cast<void**>(&ptr_), count * sizeof(T));
    if (status != cudaSuccess) {
      // A failed allocation is not sticky, but it stays the thread's last
      // error: clear it so that the next launch check does not report it.
      (void)cudaGetLastError();
      ptr_ = nullptr;
      throw std::runtime_error("cudaMalloc of " + std::to_string(count * sizeof(T)) +
                               " bytes: " + cudaGetErrorString(status));
    }
  }
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  DeviceBuffer(DeviceBuffer&& o) noexcept : ptr_(o.ptr_), count_(o.count_) {
    o.ptr_ = nullptr;
    o.count_ = 0;
  }
  DeviceBuffer& operator=(DeviceBuffer&& o) noexcept {
    std::swap(ptr_, o.ptr_);
    std::swap(count_, o.count_);
    return *this;
  }
  ~DeviceBuffer() {
    if (ptr_) cudaFree(ptr_);
  }
  T* get() const { return ptr_; }
  std::size_t size() const { return count_; }

 private:
  T* ptr_ = nullptr;
  std::size_t count_ = 0;
};

// A stream the object creates (and destroys), or one the caller lends.
class Stream {
 public:
  Stream() { QPB_CHECK(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking)); }
  explicit Stream(cudaStream_t borrowed) : s_(borrowed), owned_(borrowed == nullptr) {
    if (owned_) QPB_CHECK(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
  }
  Stream(const Stream&) = delete;
  Stream& operator=(const Stream&) = delete;
  ~Stream() {
    if (owned_) cudaStreamDestroy(s_);
  }
  operator cudaStream_t() const { return s_; }
  void sync() const { QPB_CHECK(cudaStreamSynchronize(s_)); }

 private:
  cudaStream_t s_{};
  bool owned_ = true;
};



class Graph {
 public:
  Graph(cudaGraph_t g, unsigned long long kernels) : kernels_(kernels) {
    QPB_CHECK(cudaGraphInstantiate(&exec_, g, 0));
    cudaGraphDestroy(g);
  }
  Graph(const Graph&) = delete;
  Graph& operator=(const Graph&) = delete;
  ~Graph() { cudaGraphExecDestroy(exec_); }
  void launch(cudaStream_t s) const {
    QPB_CHECK(cudaGraphLaunch(exec_, s));
    count_launches(kernels_);
  }

 private:
  cudaGraphExec_t exec_{};
  unsigned long long kernels_;
};

// Centre-origin problem arrays (QoraPhaseCU's qpcu::Problem, problem.hpp:26-31).
struct ProblemView {
  int ndim = 0;
  long long shape[3] = {0, 0, 0};
  const float* amplitude = nullptr;     // sqrt(clip(I, 0)), numel
  const std::uint8_t* mask = nullptr;   // 1 = unusable; null = none
  const std::uint8_t* support = nullptr;  // 1 = inside
  bool on_device = false;               // the arrays are device pointers
};

enum class Variant : int {
  kBatched = 0,  // `batch` starts per launch, iterations replayed from CUDA graphs
  kPlain = 1,    // one start per launch, launched directly: the in-repo baseline
  // As kBatched with fp16 storage (the reference's Variant::half and ::mixed,
  // solver.hpp:21-29, src/cuda/half.cu): kHalf keeps the iterate and the wave
  // as fp16 pairs; kMixed keeps the wave in fp16 during HIO and RAAR and runs
  // ER entirely in FP32, with an FP32 iterate throughout. Both divide the
  // amplitude by its peak; power-of-two extents only.
  kHalf = 2,
  kMixed = 3,
};

// How batched iterations run.
enum class Schedule : int {
  kAuto = 0,      // the autotuner picks (streamed groups, resident or persistent)
  kStreamed = 1,  // two (3D: four) streamed line passes per iteration, start groups as branches
  kResident = 2,  // one resident-cluster launch per chunk of iterations (square 2D, side 64/128/256)
  kPersistent = 3,  // one work-list launch per chunk of iterations (2D, sides 64/128/256)
};

struct SolverOptions {
  int starts = 1;
  int batch = 0;  // starts per launch; 0 = all (kBatched only)
  std::uint64_t seed = 0;
  const float2* start = nullptr;  // starts * numel centre-origin objects, or null
  int sync_every = 10;
  Variant variant = Variant::kBatched;
  AmpStorage amp_storage = AmpStorage::kF32;
  int device = -1;                  // CUDA ordinal; -1 = the current device
  cudaStream_t stream = nullptr;    // work stream lent by the caller; null = own stream
  bool tune = true;                 // batch == 0: let the autotuner pick starts per launch
  Schedule schedule = Schedule::kAuto;
};

// The schedule the autotuner picks for this problem and start count: the
// resident kernel or the persistent kernel (where they exist) or streamed
// passes with starts, starts/2, ..., starts/16 starts per launch (divisors
// only), timed once per (device, shape, starts, amplitude storage, variant)
// on scratch solvers and cached for the process. QPB_TUNE=0 disables it
// (streamed, all starts in one launch).
struct TunedSchedule {
  int batch;
  bool resident;
  bool persistent = false;
};
TunedSchedule tuned_schedule(const ProblemView& problem, const SolverOptions& options);

// The cached choices, for reporting: one line per tuned configuration.
std::string tuning_report();

// One recipe operation, the POD form of qpcu::Op (recipe.hpp:44).
enum OpKind : int { kOpER = 0, kOpHIO = 1, kOpRAAR = 2, kOpShrinkwrap = 3, kOpDetwinBegin = 4,
                    kOpDetwinEnd = 5 };
struct OpDesc {
  int kind;
  int n;
  float beta;
  float threshold;
  float sigma;
  int method;  // 0 max, 1 rms
  int axis;
};

using ProgressFn = void (*)(void* user, int iteration, const float* errors, int count);

// Throws Timeout when a line pass planned from `plans` gave up a bounded wait
// since the last check (the work enqueued on `stream` so far included).
void check_waits(PlanCache& plans, cudaStream_t stream);

// The recipe operation's name ("ER", "RAAR", "Shrinkwrap", ...).
const char* op_name(int kind);

// Checks shape rank and extents; returns Dims3 (2D -> {1, ny, nx}).
Dims3 dims_of(const ProblemView& p);
void validate_recipe(const OpDesc* ops, std::size_t count);
int recipe_iterations(const OpDesc* ops, std::size_t count);

// Enqueues the line passes of one array stack on a stream.
class PassRunner {
 public:
  PassRunner(Dims3 d, int ndim, PlanCache& plans);

  PassParams params(Mode mode, int axis3, int batch) const;
  void launch(Mode mode, int axis3, PassParams p, cudaStream_t s) const;
  int outer() const { return ndim_ == 2 ? 1 : 0; }
  bool has_mid() const { return ndim_ == 3; }
  Dims3 dims() const { return d_; }
  // Polls a staged wait makes before giving up (kMaxWaitTries by default), and
  // the timeout tests' fault injection (staged copies left out); both apply to
  // passes whose parameters are made afterwards.
  void set_wait(int tries, bool starve) {
    wait_tries_ = tries;
    starve_ = starve;
  }

 private:
  Dims3 d_;
  int ndim_;
  const LinePlan* plans_[3];
  int* wait_failures_;
  int wait_tries_;
  bool starve_ = false;
};

// Line plans shared by the single operators and the problem set-up, one cache
// per device for the process.
PlanCache& operator_plans();

// DeviceSelect makes `requested` (>= 0) the calling thread's device before any
// allocation and remembers the device in use.
struct DeviceSelect {
  int device = 0;
  explicit DeviceSelect(int requested) {
    if (requested >= 0) QPB_CHECK(cudaSetDevice(requested));
    QPB_CHECK(cudaGetDevice(&device));
  }
};

// Several problems of one shape may share a solver: options.starts starts per
// problem, problem q's starts at q * starts, each with its own amplitude,
// mask, support and error normalisation, random starts keyed as if the
// problem ran alone.
class Solver {
 public:
  Solver(const ProblemView& problem, const SolverOptions& options);
  Solver(const std::vector<ProblemView>& problems, const SolverOptions& options);
  ~Solver();
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;

  void run(const OpDesc* ops, std::size_t count);
  // New problems of the same shape and count in the same solver: buffers and
  // captured graphs are kept, the iterate, supports and error histories start
  // afresh from `seed` or the given starts (as construction does).
  void reset(const std::vector<ProblemView>& problems, std::uint64_t seed, const float2* start);
  std::size_t error_count() const { return errors_.empty() ? 0 : errors_[0].size(); }
  int starts() const { return starts_; }
  int problems() const { return problems_; }
  bool resident() const { return resident_; }
  bool persistent() const { return persistent_; }
  int batch() const { return batch_; }
  long long numel() const { return n_; }
  int ndim() const { return ndim_; }
  int device() const { return select_.device; }
  cudaStream_t stream() const { return stream_; }
  // objects: starts * numel complex64; supports: starts * numel; errors: starts * error_count().
  void results(float2* objects, std::uint8_t* supports, float* errors);
  // As results(), each problem's block of starts to its own host place:
  // objects[q] (starts-per-problem * numel complex64), supports[q], errors[q]
  // (starts-per-problem * error_count()); a null array, or a null entry, skips.
  void results_per_problem(float2* const* objects, std::uint8_t* const* supports,
                           float* const* errors);
  // As results(), objects and supports written to device memory (centre-origin)
  // on the solver's stream, which is synchronised before returning; errors on the host.
  void results_device(float2* objects, std::uint8_t* supports, float* errors);
  void set_progress(ProgressFn fn, void* user) {
    progress_ = fn;
    progress_user_ = user;
  }
  // Launches each pass of an iteration `iterations` times back to back between
  // two CUDA events; ms[p] receives the mean time per launch of pass p.
  // Returns the number of passes per iteration (at most 8). Changes the state.
  int profile_passes(int iterations, double* ms);

  // The steps of run(), for a driver that captures the chunks of several
  // solvers on one stream into one graph (BatchSolver):
  //   begin_run; per op: iterations -> begin_iterate, then per chunk
  //   chunk_length / prepare_branches / enqueue_chunk_body (captured) / end_chunk;
  //   other ops -> apply; finally end_run.
  void begin_run(const OpDesc* ops, std::size_t count);
  void begin_iterate(Coefficients c);
  int chunk_length(int remaining) const;
  void prepare_branches();
  void enqueue_chunk_body(int len, cudaStream_t s);
  void end_chunk(int len);
  void apply(const OpDesc& o);
  void end_run();
  // The latest error of every start (after at least one iteration of this run).
  std::vector<float> latest_errors();
  bool batched() const { return options_.variant != Variant::kPlain; }
  bool wave_half() const { return wave_half_; }
  bool fp16_wave_variant() const {
    return options_.variant == Variant::kHalf || options_.variant == Variant::kMixed;
  }
  // Bounded waits: `tries` polls before a staged wait gives up; `starve`
  // leaves the staged copies out so that every such wait runs out (the fault
  // injection of the timeout tests; results are invalid and run() reports
  // Timeout). Captured graphs are dropped so that the next chunks pick it up.
  void set_wait(int tries, bool starve);

 private:
  // The iterate of group g in its storage: complex64, or fp16 pairs (half variant).
  float2* x(int g) const {
    if (iter_half_) {
      return reinterpret_cast<float2*>(xh_.get() + static_cast<std::size_t>(g) * batch_ * n_);
    }
    return x_.get() + static_cast<std::size_t>(g) * batch_ * n_;
  }
  // The wave of group g in its storage (fp16 pairs pack into the buffer's first half).
  float2* w(int g) const {
    if (wave_half_) {
      return reinterpret_cast<float2*>(reinterpret_cast<std::uint32_t*>(w_.get()) +
                                       static_cast<std::size_t>(g) * batch_ * n_);
    }
    return w_.get() + static_cast<std::size_t>(g) * batch_ * n_;
  }
  std::uint8_t* support(int g) const {
    return support_.get() + static_cast<std::size_t>(g) * batch_ * n_;
  }
  PassParams base(Mode mode, int axis3, int g) const;

  void load(const std::vector<ProblemView>& problems, std::uint64_t seed, const float2* start);
  void enqueue_iteration(int g, cudaStream_t s);
  void enqueue_chunk(int len, cudaStream_t s);  // resident: `len` iterations in one launch
  // w = FFT_inner(x) for `count` starts from group g's first one
  void enqueue_establish(int g, int count);
  void establish_wave();
  void iterate(int count, Coefficients c);
  void shrinkwrap(const OpDesc& o);
  void detwin_begin(int axis);
  void detwin_end();
  void collect_errors(int iterations);
  // The power-of-two register-resident or column pass for every pass an fp16
  // variant launches; InvalidArgument otherwise.
  void require_fp16_passes() const;
  // The complex64, unscaled iterate (centre-origin or FFT order as x_ holds
  // it) into `out` (starts * numel): widened from fp16 and multiplied back by
  // each problem's amplitude peak where the variant stores it so.
  void iterate_f32(float2* out);
  void report();
  float to_error(double num, int start) const;

  Dims3 d_;
  int ndim_;
  long long n_;
  int problems_;
  int spp_;  // starts per problem
  int starts_;
  int batch_;
  int groups_;
  SolverOptions options_;
  DeviceSelect select_;  // before any allocation; every later call re-selects it
  PlanCache plans_;
  Stream stream_;
  PassRunner runner_;
  std::vector<double> energies_;     // usable energy per problem
  long long amp_stride_ = 0;         // elements between problems' amplitudes in amp_
  DeviceBuffer<unsigned char> amp_;  // signed amplitude in the chosen storage
  DeviceBuffer<float> amp_f_;        // FP32 FFT-order amplitude, for the random starts
  DeviceBuffer<unsigned char> prep_;  // problem set-up: scratch, and host arrays staged
  int amp_tiled_ = 0;                // amp_ in the modulus pass's CTA order (kAmpTiled*)
  bool resident_ = false;            // iterations run by the resident kernel
  bool persistent_ = false;          // iterations run by the persistent kernel
  DeviceBuffer<unsigned> work_;      // the persistent kernel's work-list words
  DeviceBuffer<float2> x_;
  DeviceBuffer<std::uint32_t> xh_;   // the half variant's fp16 iterate (one __half2 per element)
  DeviceBuffer<float2> w_;           // the wave; fp16 pairs in its first half while wave_half_
  DeviceBuffer<float> peaks_;        // per problem: the amplitude peak an fp16 variant divides by
  std::vector<float> amp_scale_;     // host copy of peaks_ (1 without amplitude scaling)
  bool wave_half_ = false;           // the wave is stored as fp16 pairs
  bool iter_half_ = false;           // the iterate is stored as fp16 pairs (xh_)
  DeviceBuffer<std::uint8_t> support_;
  DeviceBuffer<std::uint8_t> saved_;
  DeviceBuffer<LevelAcc> level_;
  DeviceBuffer<unsigned long long> moments_;
  DeviceBuffer<Ctrl> ctrl_;
  DeviceBuffer<int> counters_;
  DeviceBuffer<double> errs_;
  int capacity_ = 0;
  bool wave_valid_ = false;
  std::map<int, std::unique_ptr<Graph>> graphs_;  // by 2 * chunk length + wave_half_
  // Captured graphs run start groups as parallel branches, one stream each.
  std::vector<std::unique_ptr<Stream>> branches_;
  std::vector<cudaEvent_t> branch_events_;
  std::vector<std::vector<float>> errors_;
  std::vector<double> host_errs_;
  int iteration_ = 0;
  int run_iterations_ = 0;
  ProgressFn progress_ = nullptr;
  void* progress_user_ = nullptr;
};

// ---- single operators on centre-origin arrays (operators.hpp:13-33)
// Replaces obj (numel complex64, centre-origin) by P_M obj; returns the Fourier
// error of the input.
float modulus_project(const ProblemView& problem, float2* obj, AmpStorage storage);
void support_project_host(const std::uint8_t* support, float2* obj, long long count);
void gaussian_blur(const float* image, int ndim, const long long* shape, float sigma, float* out);
// aligned_error (metrics.cpp:17-86) of `batch` candidates a[b] (numel complex64
// each) against one reference, on the device; out[b] = the smaller of the
// direct and twin errors. Host arrays.
void aligned_error(const float2* a, const float2* reference, int ndim, const long long* shape,
                   int batch, float* out);
// The same alignment, also applied: errors[b] as aligned_error (may be null),
// aligned[b] = object b (or its twin, whichever fits better) translated and
// phase-rotated onto the reference (batch * numel, may be null), mean = their
// average (numel, may be null). Host arrays.
void align(const float2* a, const float2* reference, int ndim, const long long* shape, int batch,
           float* errors, float2* aligned, float2* mean);
// simulate_intensity (problem.cpp:90-99): |centred unitary FFT(object)|^2 of a
// centre-origin complex64 object, FFT on the device. Host arrays.
void simulate_intensity(const float2* object, int ndim, const long long* shape, float* out);
// half_support on the device (problem.cpp:101-127), centre-origin in and out.
void half_support(const std::uint8_t* support, int ndim, const long long* shape, int axis,
                  std::uint8_t* out);

}  // namespace qpb
