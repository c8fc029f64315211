#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <execinfo.h>
#include <unistd.h>

#include <csignal>

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "bulk_copy.cuh"
#include "column_pass.cuh"
#include "device_setup.cuh"
#include "fast_pass.cuh"
#include "nvtx_range.hpp"
#include "persistent.cuh"
#include "resident.cuh"
#include "solver.hpp"

namespace qpb {

namespace {
std::atomic<unsigned long long> g_launches{0};
}  // namespace

void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
unsigned long long launches() { return g_launches.load(std::memory_order_relaxed); }

namespace {
void crash_handler(int sig) {
  void* frames[64];
  const int n = backtrace(frames, 64);
  const char msg[] = "[qpb] fatal signal, native backtrace:\n";
  (void)!write(2, msg, sizeof(msg) - 1);
  backtrace_symbols_fd(frames, n, 2);
  signal(sig, SIG_DFL);
  raise(sig);
}
}  // namespace

// QPB_TRACE=1 logs host-side steps; any non-zero value (e.g. "backtrace") also
// prints a native backtrace on SIGSEGV.
bool tracing() {
  static const bool on = [] {
    const char* v = std::getenv("QPB_TRACE");
    const bool enabled = v && *v && std::strcmp(v, "0") != 0;
    if (enabled) signal(SIGSEGV, crash_handler);
    return enabled && std::strcmp(v, "1") == 0;
  }();
  return on;
}

namespace {
// Installs the crash handler at load time when QPB_TRACE asks for it.
const bool g_trace_init = (tracing(), true);
}  // namespace

void trace(const char* fmt, ...) {
  if (!tracing()) return;
  std::va_list args;
  va_start(args, fmt);
  std::fputs("[qpb] ", stderr);
  std::vfprintf(stderr, fmt, args);
  std::fputc('\n', stderr);
  std::fflush(stderr);
  va_end(args);
}

void check_waits(PlanCache& plans, cudaStream_t stream) {
  if (const int failed = plans.take_wait_failures(stream)) {
    throw Timeout(std::to_string(failed) +
                  " line-pass CTAs gave up waiting for their staged inputs; results are invalid");
  }
}

namespace {

// out[i] = in[(i + off(n)) mod n] per axis, src/core/layout.hpp:71-88.
template <class T>
std::vector<T> host_roll(const T* in, Dims3 d, bool to_fft_order) {
  auto off = [&](int len) { return to_fft_order ? len / 2 : len - len / 2; };
  const int o0 = off(d.d0), o1 = off(d.d1), o2 = off(d.d2);
  std::vector<T> out(static_cast<std::size_t>(d.n()));
  std::size_t i = 0;
  for (int z = 0; z < d.d0; ++z) {
    const int sz = (z + o0) % d.d0;
    for (int y = 0; y < d.d1; ++y) {
      const std::size_t row = (static_cast<std::size_t>(sz) * d.d1 + (y + o1) % d.d1) * d.d2;
      for (int x = 0; x < d.d2; ++x) out[i++] = in[row + (x + o2) % d.d2];
    }
  }
  return out;
}

// Signed amplitude (-1 on masked pixels) in the requested storage type.
std::vector<unsigned char> signed_amplitude(const std::vector<float>& amp,
                                            const std::vector<std::uint8_t>& mask,
                                            AmpStorage storage) {
  const std::size_t n = amp.size();
  std::vector<unsigned char> out;
  switch (storage) {
    case AmpStorage::kF32: {
      out.resize(n * sizeof(float));
      auto* p = reinterpret_cast<float*>(out.data());
      for (std::size_t i = 0; i < n; ++i) p[i] = mask[i] ? -1.0f : amp[i];
      break;
    }
    case AmpStorage::kF16: {
      out.resize(n * sizeof(__half));
      auto* p = reinterpret_cast<__half*>(out.data());
      for (std::size_t i = 0; i < n; ++i) p[i] = __float2half_rn(mask[i] ? -1.0f : amp[i]);
      break;
    }
    case AmpStorage::kBF16: {
      out.resize(n * sizeof(__nv_bfloat16));
      auto* p = reinterpret_cast<__nv_bfloat16*>(out.data());
      for (std::size_t i = 0; i < n; ++i) p[i] = __float2bfloat16_rn(mask[i] ? -1.0f : amp[i]);
      break;
    }
  }
  return out;
}

double usable_energy(const std::vector<float>& amp, const std::vector<std::uint8_t>& mask) {
  double e = 0.0;
  for (std::size_t i = 0; i < amp.size(); ++i) {
    if (!mask[i]) e += static_cast<double>(amp[i]) * amp[i];
  }
  return e;
}

template <class T>
DeviceBuffer<T> upload(const std::vector<T>& host, cudaStream_t s) {
  DeviceBuffer<T> d(host.size());
  QPB_CHECK(cudaMemcpyAsync(d.get(), host.data(), host.size() * sizeof(T), cudaMemcpyHostToDevice, s));
  QPB_CHECK(cudaStreamSynchronize(s));
  return d;
}

int axis_stride(Dims3 d, int axis3) {
  return axis3 == 2 ? 1 : axis3 == 1 ? d.d2 : d.d1 * d.d2;
}

int axis_len(Dims3 d, int axis3) { return axis3 == 0 ? d.d0 : axis3 == 1 ? d.d1 : d.d2; }

}  // namespace

Dims3 dims_of(const ProblemView& p) {
  if (p.ndim != 2 && p.ndim != 3) {
    throw InvalidArgument("problem shape must be 2D or 3D, got ndim=" + std::to_string(p.ndim));
  }
  for (int a = 0; a < p.ndim; ++a) {
    if (p.shape[a] < 1) throw InvalidArgument("shape has a zero-length axis");
    if (p.shape[a] > kMaxLine) {
      throw InvalidArgument("axis length " + std::to_string(p.shape[a]) +
                            " exceeds the supported maximum " + std::to_string(kMaxLine));
    }
  }
  if (p.ndim == 2) return {1, static_cast<int>(p.shape[0]), static_cast<int>(p.shape[1])};
  return {static_cast<int>(p.shape[0]), static_cast<int>(p.shape[1]), static_cast<int>(p.shape[2])};
}

// src/core/recipe.cpp:30-61, plus the axis check half_support makes (problem.cpp:104-106).
void validate_recipe(const OpDesc* ops, std::size_t count) {
  if (count == 0) throw InvalidArgument("recipe is empty");
  bool in_detwin = false;
  for (std::size_t i = 0; i < count; ++i) {
    const OpDesc& o = ops[i];
    switch (o.kind) {
      case kOpER:
        if (o.n < 1) throw InvalidArgument("ER needs n >= 1");
        break;
      case kOpHIO:
        if (o.n < 1) throw InvalidArgument("HIO needs n >= 1");
        break;
      case kOpRAAR:
        if (o.n < 1) throw InvalidArgument("RAAR needs n >= 1");
        break;
      case kOpShrinkwrap:
        if (!(o.threshold > 0.0f) || !(o.sigma >= 0.0f)) {
          throw InvalidArgument("Shrinkwrap needs threshold > 0, sigma >= 0");
        }
        if (o.method != 0 && o.method != 1) throw InvalidArgument("unknown shrinkwrap method");
        break;
      case kOpDetwinBegin:
        if (in_detwin) throw InvalidArgument("nested detwin");
        in_detwin = true;
        break;
      case kOpDetwinEnd:
        if (!in_detwin) throw InvalidArgument("DetwinEnd without DetwinBegin");
        in_detwin = false;
        break;
      default:
        throw InvalidArgument("unknown recipe operation " + std::to_string(o.kind));
    }
  }
  if (in_detwin) throw InvalidArgument("DetwinBegin without DetwinEnd");
}

int recipe_iterations(const OpDesc* ops, std::size_t count) {
  long long total = 0;
  for (std::size_t i = 0; i < count; ++i) {
    if (ops[i].kind == kOpER || ops[i].kind == kOpHIO || ops[i].kind == kOpRAAR) total += ops[i].n;
  }
  if (total > (1LL << 30)) throw InvalidArgument("recipe has too many iterations");
  return static_cast<int>(total);
}

// ------------------------------------------------------------------ PassRunner
PassRunner::PassRunner(Dims3 d, int ndim, PlanCache& plans)
    : d_(d), ndim_(ndim), wait_failures_(plans.wait_failures()), wait_tries_(kMaxWaitTries) {
  configure_line_passes();
  for (int a = 0; a < 3; ++a) {
    plans_[a] = (ndim == 2 && a == 0) ? nullptr : &plans.get(axis_len(d, a));
  }
}

PassParams PassRunner::params(Mode mode, int axis3, int batch) const {
  (void)mode;
  PassParams p{};
  const LinePlan& plan = *plans_[axis3];
  p.n = d_.n();
  p.L = plan.length;
  p.S = axis_stride(d_, axis3);
  p.lines_per_start = static_cast<int>(p.n / p.L);
  p.lines = batch * p.lines_per_start;
  p.lpc = choose_lpc(p.L, p.S, p.lines_per_start);
  p.stages = plan.stages;
  for (int s = 0; s < plan.stages; ++s) p.radix[s] = plan.radix[s];
  p.twiddle = plan.twiddle;
  p.stage_twiddle = plan.stage_twiddle;
  p.scale = 1.0f / std::sqrt(static_cast<float>(p.n));
  p.amp_stride = 0;
  p.starts_per_problem = 1;
  p.wait_tries = wait_tries_;
  p.wait_failures = wait_failures_;
  p.starve = starve_ ? 1 : 0;
  return p;
}

void PassRunner::launch(Mode mode, int axis3, PassParams p, cudaStream_t s) const {
  (void)axis3;
  launch_line_pass(mode, p, s);
}

// ---------------------------------------------------------------------- Solver
Solver::Solver(const ProblemView& problem, const SolverOptions& options)
    : Solver(std::vector<ProblemView>{problem}, options) {}

Solver::Solver(const std::vector<ProblemView>& problems, const SolverOptions& options)
    : d_(dims_of(problems.at(0))),
      ndim_(problems[0].ndim),
      n_(d_.n()),
      problems_(static_cast<int>(problems.size())),
      spp_(options.starts),
      starts_(options.starts * static_cast<int>(problems.size())),
      batch_(1),
      groups_(1),
      options_(options),
      select_(options.device),
      stream_(options.stream),
      runner_(d_, ndim_, plans_) {
  if (options.starts < 1) throw InvalidArgument("starts must be >= 1");
  if (options.sync_every < 1) throw InvalidArgument("sync_every must be >= 1");
  if (options.batch < 0 || (options.batch > 0 && starts_ % options.batch != 0)) {
    throw InvalidArgument("batch must divide starts");
  }
  for (const ProblemView& q : problems) {
    if (!q.amplitude || !q.support) {
      throw InvalidArgument("problem arrays do not match its shape; build it with make_problem");
    }
    const Dims3 dq = dims_of(q);
    if (q.ndim != ndim_ || dq.d0 != d_.d0 || dq.d1 != d_.d1 || dq.d2 != d_.d2) {
      throw InvalidArgument("problems of one solver must share a shape");
    }
  }
  const ProblemView& problem = problems[0];
  if (fp16_wave_variant()) {
    // The reference's fp16 variants need power-of-two extents (its fp16
    // cuFFT, src/cuda/cuda_solver.cu:74-80); here the fp16 storage runs on the
    // register-resident and column passes, which take 16..1024 points.
    if (options.amp_storage != AmpStorage::kF32) {
      throw InvalidArgument("the half and mixed variants keep the amplitude in FP32");
    }
    for (int a = 0; a < ndim_; ++a) {
      const long long len = problem.shape[a];
      if (len < 16 || len > 1024 || (len & (len - 1)) != 0) {
        throw InvalidArgument(
            "the half and mixed variants need power-of-two extents of 16..1024 (fp16 storage)");
      }
    }
    if (options.schedule == Schedule::kResident || options.schedule == Schedule::kPersistent) {
      throw InvalidArgument("the half and mixed variants run the streamed passes, not the "
                            "resident or persistent schedule");
    }
  }
  const bool persistent_ok = options.variant == Variant::kBatched &&
                             persistent_supports(problem.ndim, d_.d1, d_.d2);
  if (options.schedule == Schedule::kPersistent && !persistent_ok) {
    throw InvalidArgument("the persistent schedule runs batched complex64 starts of 2D problems "
                          "with sides of 64, 128 or 256");
  }
  const bool resident_ok = resident_supports(problem.ndim, d_.d1, d_.d2) && !fp16_wave_variant();
  if (options.schedule == Schedule::kResident) {
    if (options.variant == Variant::kPlain) {
      throw InvalidArgument("the resident schedule runs batched starts only");
    }
    if (!resident_ok) {
      throw InvalidArgument("the resident schedule needs a square 2D problem of side 64, 128 or 256");
    }
  }
  if (options.variant == Variant::kPlain) {
    batch_ = 1;
  } else if (options.schedule == Schedule::kResident) {
    resident_ = true;
  } else if (options.schedule == Schedule::kPersistent) {
    persistent_ = true;
  } else if (options.batch) {
    batch_ = options.batch;
  } else if (options.tune) {
    // Tuned on the first problem with every start: the work is the same.
    SolverOptions o = options;
    o.starts = starts_;
    if (!resident_ok && !persistent_ok) o.schedule = Schedule::kStreamed;
    const TunedSchedule t = tuned_schedule(problem, o);
    batch_ = t.batch;
    resident_ = t.resident && resident_ok;
    persistent_ = t.persistent && persistent_ok;
  } else {
    batch_ = starts_;
  }
  if (resident_ || persistent_) batch_ = starts_;
  groups_ = starts_ / batch_;
  if (resident_) configure_resident();
  if (persistent_) {
    configure_persistent();
    work_ = DeviceBuffer<unsigned>(static_cast<std::size_t>(persistent_work_words(starts_)));
  }
  iter_half_ = options.variant == Variant::kHalf;
  wave_half_ = fp16_wave_variant();
  if (fp16_wave_variant()) require_fp16_passes();
  options_.start = nullptr;
  amp_stride_ = problems_ > 1 ? n_ : 0;

  // The modulus pass reads its amplitude tile by one bulk copy when the
  // amplitude is stored in its CTA order: line-major for the TMA column pass
  // (where it is preferred, and always for the persistent kernel's column
  // tiles), element-major for the register-resident pass.
  PassParams mod = runner_.params(Mode::kMod, runner_.outer(), batch_);
  mod.amp_tiled = kAmpTiledLines;
  if (!resident_ && (persistent_ ? column_pass_lines(mod, Mode::kMod) > 0
                                 : column_pass_preferred(mod, Mode::kMod))) {
    amp_tiled_ = kAmpTiledLines;
  } else if (!resident_ && fast_pass_lines(mod) > 0 && mod.S > 1) {
    amp_tiled_ = kAmpTiledElements;
  }
  const std::size_t total = static_cast<std::size_t>(starts_) * n_;
  const std::size_t elem = options.amp_storage == AmpStorage::kF32 ? 4 : 2;
  amp_ = DeviceBuffer<unsigned char>(static_cast<std::size_t>(problems_) * n_ * elem);
  amp_f_ = DeviceBuffer<float>(static_cast<std::size_t>(problems_) * n_);
  support_ = DeviceBuffer<std::uint8_t>(total);
  x_ = DeviceBuffer<float2>(total);
  if (iter_half_) xh_ = DeviceBuffer<std::uint32_t>(total);
  if (fp16_wave_variant()) peaks_ = DeviceBuffer<float>(static_cast<std::size_t>(problems_));
  w_ = DeviceBuffer<float2>(total);
  saved_ = DeviceBuffer<std::uint8_t>(total);
  level_ = DeviceBuffer<LevelAcc>(static_cast<std::size_t>(starts_));
  moments_ = DeviceBuffer<unsigned long long>(2 * static_cast<std::size_t>(starts_));
  ctrl_ = DeviceBuffer<Ctrl>(1);
  counters_ = DeviceBuffer<int>(static_cast<std::size_t>(groups_));
  load(problems, options.seed, options.start);
}

void Solver::reset(const std::vector<ProblemView>& problems, std::uint64_t seed,
                   const float2* start) {
  if (static_cast<int>(problems.size()) != problems_) {
    throw InvalidArgument("reset needs as many problems as the solver was built for");
  }
  for (const ProblemView& q : problems) {
    const Dims3 dq = dims_of(q);
    if (q.ndim != ndim_ || dq.d0 != d_.d0 || dq.d1 != d_.d1 || dq.d2 != d_.d2) {
      throw InvalidArgument("reset needs problems of the solver's shape");
    }
    if (!q.amplitude || !q.support) {
      throw InvalidArgument("problem arrays do not match its shape; build it with make_problem");
    }
  }
  load(problems, seed, start);
}

// Problems into the solver's buffers: per problem the FFT-order amplitude,
// mask and support, the signed amplitude in the storage type (in the modulus
// pass's CTA order when that pass tiles it, so each CTA stages its tile with
// one bulk copy) and the usable energy, all prepared on the device (host
// arrays are staged there first); then the starts, drawn or given. The
// captured graphs stay valid: every buffer keeps its address.
void Solver::load(const std::vector<ProblemView>& problems, std::uint64_t seed,
                  const float2* start) {
  PassParams mod = runner_.params(Mode::kMod, runner_.outer(), batch_);
  mod.amp_tiled = amp_tiled_;
  const int lines = amp_tiled_ == kAmpTiledLines     ? column_pass_lines(mod, Mode::kMod)
                    : amp_tiled_ == kAmpTiledElements ? fast_pass_lines(mod)
                                                      : 0;
  const std::size_t elem = options_.amp_storage == AmpStorage::kF32 ? 4 : 2;
  const std::size_t total = static_cast<std::size_t>(starts_) * n_;
  const bool on_device = problems[0].on_device;
  for (const ProblemView& q : problems) {
    if (q.on_device != on_device) throw InvalidArgument("problems mix host and device arrays");
  }
  // prep_: the problems' energies, then per problem its set-up scratch and,
  // for host arrays, the staged amplitude, mask and support
  const auto n = static_cast<std::size_t>(n_);
  auto round256 = [](std::size_t b) { return (b + 255) / 256 * 256; };
  const std::size_t head = round256(static_cast<std::size_t>(problems_) * sizeof(double));
  const std::size_t scratch = prepare_scratch_bytes(n_);
  const std::size_t amp_bytes = round256(n * sizeof(float));
  const std::size_t staged = on_device ? 0 : amp_bytes + 2 * round256(n);
  const std::size_t per_problem = scratch + staged;
  const std::size_t bytes = head + static_cast<std::size_t>(problems_) * per_problem;
  if (prep_.size() < bytes) {
    prep_ = DeviceBuffer<unsigned char>();
    prep_ = DeviceBuffer<unsigned char>(bytes);
  }
  auto* energies = reinterpret_cast<double*>(prep_.get());
  for (int q = 0; q < problems_; ++q) {
    ProblemView v = problems[q];
    unsigned char* region = prep_.get() + head + static_cast<std::size_t>(q) * per_problem;
    if (!on_device) {
      unsigned char* stage = region + scratch;
      auto* amp = reinterpret_cast<float*>(stage);
      std::uint8_t* mask = stage + amp_bytes;
      std::uint8_t* sup = mask + round256(n);
      QPB_CHECK(cudaMemcpyAsync(amp, v.amplitude, n * sizeof(float), cudaMemcpyHostToDevice,
                                stream_));
      if (v.mask) {
        QPB_CHECK(cudaMemcpyAsync(mask, v.mask, n, cudaMemcpyHostToDevice, stream_));
      }
      QPB_CHECK(cudaMemcpyAsync(sup, v.support, n, cudaMemcpyHostToDevice, stream_));
      v.amplitude = amp;
      v.mask = v.mask ? mask : nullptr;
      v.support = sup;
      v.on_device = true;
    }
    prepare_problem_device(v, d_, options_.amp_storage, mod.L, mod.S, lines,
                           amp_tiled_ == kAmpTiledLines,
                           amp_f_.get() + static_cast<std::size_t>(q) * n_,
                           amp_.get() + static_cast<std::size_t>(q) * n_ * elem,
                           support_.get() + static_cast<std::size_t>(q) * spp_ * n_, region,
                           energies + q, fp16_wave_variant() ? peaks_.get() + q : nullptr,
                           stream_);
  }
  energies_.assign(static_cast<std::size_t>(problems_), 0.0);
  QPB_CHECK(cudaMemcpyAsync(energies_.data(), energies, energies_.size() * sizeof(double),
                            cudaMemcpyDeviceToHost, stream_));
  amp_scale_.assign(static_cast<std::size_t>(problems_), 1.0f);
  if (fp16_wave_variant()) {
    QPB_CHECK(cudaMemcpyAsync(amp_scale_.data(), peaks_.get(), amp_scale_.size() * sizeof(float),
                              cudaMemcpyDeviceToHost, stream_));
  }
  QPB_CHECK(cudaMemsetAsync(x_.get(), 0, total * sizeof(float2), stream_));
  QPB_CHECK(cudaMemsetAsync(counters_.get(), 0, groups_ * sizeof(int), stream_));
  const Ctrl ctrl{nullptr, 0, 0.0f, 0.0f, counters_.get()};
  set_ctrl(ctrl_.get(), ctrl, stream_);
  for (int q = 0; q < problems_; ++q) {
    std::uint8_t* first = support_.get() + static_cast<std::size_t>(q) * spp_ * n_;
    // the first start's support to the others, doubling the copied block
    for (int have = 1; have < spp_;) {
      const int take = std::min(have, spp_ - have);
      QPB_CHECK(cudaMemcpyAsync(first + static_cast<std::size_t>(have) * n_, first,
                                static_cast<std::size_t>(take) * n_, cudaMemcpyDeviceToDevice,
                                stream_));
      have += take;
    }
  }
  stream_.sync();
  errors_.assign(static_cast<std::size_t>(starts_), {});
  iteration_ = 0;
  run_iterations_ = 0;

  // The starts are made in complex64 (x_, and the wave buffer as complex64),
  // as the reference makes an fp16 variant's starts in FP32 before rounding
  // them (src/cuda/cuda_solver.cu:125-140); the storage flags are restored
  // below, and an fp16 iterate is rounded from x_ at the end.
  const bool wave_half = wave_half_;
  const bool iter_half = iter_half_;
  wave_half_ = false;
  iter_half_ = false;
  if (start) {
    // Given starts, centre-origin: to FFT order, cut to the support
    // (cpu_solver.cpp:37-41), brought into the scale of an fp16 variant's
    // amplitude (divided by its peak, as test_cuda.cpp:192-205 requires).
    QPB_CHECK(cudaMemcpyAsync(w_.get(), start, total * sizeof(float2), cudaMemcpyDefault,
                              stream_));
    roll<float2>(w_.get(), x_.get(), d_, starts_, true, stream_);
    support_project(x_.get(), support_.get(), n_, starts_, stream_);
    if (fp16_wave_variant()) {
      const std::size_t block = static_cast<std::size_t>(spp_) * n_;
      for (int q = 0; q < problems_; ++q) {
        scale_complex(x_.get() + q * block, static_cast<long long>(block),
                      1.0f / amp_scale_[static_cast<std::size_t>(q)], stream_);
      }
    }
    wave_valid_ = false;
  } else {
    // Random phases on the measured amplitude, inverse transform, cut to the
    // support (kernels.cpp:104-117): the inverse's last pass is an ER update.
    // A batched solver draws every start in one launch per pass (each start
    // keyed by its global index, as in its own group); the plain variant one
    // start per launch.
    const bool together = batched();
    const int chunks = together ? 1 : groups_;
    const int count = together ? starts_ : batch_;
    auto params = [&](Mode mode, int axis3, int g) {
      PassParams p = base(mode, axis3, g);
      p.lines = runner_.params(mode, axis3, count).lines;
      return p;
    };
    for (int g = 0; g < chunks; ++g) {
      random_wave(w(g), amp_f_.get(), amp_stride_, spp_, n_, count, seed,
                  static_cast<std::uint64_t>(g) * batch_, stream_);
      const int outer = runner_.outer();
      runner_.launch(Mode::kInv, outer, params(Mode::kInv, outer, g), stream_);
      if (runner_.has_mid()) runner_.launch(Mode::kInv, 1, params(Mode::kInv, 1, g), stream_);
      PassParams u = params(Mode::kUpd, 2, g);
      u.coef_from_ctrl = 0;
      u.coef_a = 0.0f;
      u.coef_b = 0.0f;
      u.bump_counter = 0;
      runner_.launch(Mode::kUpd, 2, u, stream_);
      if (runner_.has_mid()) runner_.launch(Mode::kFwd, 1, params(Mode::kFwd, 1, g), stream_);
    }
    wave_valid_ = true;
  }
  wave_half_ = wave_half;
  iter_half_ = iter_half;
  if (iter_half_) to_half(x_.get(), xh_.get(), static_cast<long long>(total), stream_);
  if (wave_half_) wave_valid_ = false;  // the complex64 wave of the starts is not the fp16 one
  if (!wave_valid_) establish_wave();
  stream_.sync();
}

Solver::~Solver() {
  cudaStreamSynchronize(stream_);
  graphs_.clear();
  for (cudaEvent_t e : branch_events_) cudaEventDestroy(e);
}

PassParams Solver::base(Mode mode, int axis3, int g) const {
  PassParams p = runner_.params(mode, axis3, batch_);
  p.w = w(g);
  p.x = x(g);
  p.amp = amp_.get();
  p.support = support(g);
  p.ctrl = ctrl_.get();
  p.level = level_.get();
  p.group = g;
  p.start0 = g * batch_;
  p.starts_total = starts_;
  p.coef_from_ctrl = 1;
  p.bump_counter = 1;
  p.amp_storage = options_.amp_storage;
  p.amp_tiled = mode == Mode::kMod ? amp_tiled_ : 0;
  p.amp_stride = amp_stride_;
  p.starts_per_problem = spp_;
  p.wave_half = wave_half_ ? 1 : 0;
  p.iter_half = iter_half_ ? 1 : 0;
  return p;
}

void Solver::enqueue_establish(int g, int count) {
  PassParams first = base(Mode::kFwdFromX, 2, g);
  first.lines = runner_.params(Mode::kFwdFromX, 2, count).lines;
  runner_.launch(Mode::kFwdFromX, 2, first, stream_);
  if (runner_.has_mid()) {
    PassParams mid = base(Mode::kFwd, 1, g);
    mid.lines = runner_.params(Mode::kFwd, 1, count).lines;
    runner_.launch(Mode::kFwd, 1, mid, stream_);
  }
}

// A batched solver's starts in one launch per axis, whatever its groups; the
// plain variant one start per launch like the rest of its iteration.
void Solver::establish_wave() {
  if (batched()) {
    enqueue_establish(0, starts_);
  } else {
    for (int g = 0; g < groups_; ++g) enqueue_establish(g, batch_);
  }
  wave_valid_ = true;
}

// One iteration of group g (cpu_solver.cpp:84-89): forward FFT, modulus with
// the error, inverse FFT, update; the x-axis forward of the new iterate is
// folded into the update pass.
void Solver::enqueue_iteration(int g, cudaStream_t s) {
  const int outer = runner_.outer();
  runner_.launch(Mode::kMod, outer, base(Mode::kMod, outer, g), s);
  if (runner_.has_mid()) runner_.launch(Mode::kInv, 1, base(Mode::kInv, 1, g), s);
  runner_.launch(Mode::kUpd, 2, base(Mode::kUpd, 2, g), s);
  if (runner_.has_mid()) runner_.launch(Mode::kFwd, 1, base(Mode::kFwd, 1, g), s);
}

void Solver::enqueue_chunk(int len, cudaStream_t s) {
  ResidentParams p{};
  p.x = x_.get();
  p.w = w_.get();
  p.amp = amp_.get();
  p.amp_stride = amp_stride_;
  p.starts_per_problem = spp_;
  p.support = support_.get();
  p.ctrl = ctrl_.get();
  p.twiddle = runner_.params(Mode::kFwd, 2, starts_).stage_twiddle;
  p.group = 0;
  p.start0 = 0;
  p.starts_total = starts_;
  p.iterations = len;
  p.scale = 1.0f / static_cast<float>(d_.d2);
  p.amp_storage = options_.amp_storage;
  launch_resident(p, d_.d2, starts_, s);
}

void Solver::begin_run(const OpDesc* ops, std::size_t count) {
  validate_recipe(ops, count);
  for (std::size_t i = 0; i < count; ++i) {
    if (ops[i].kind == kOpDetwinBegin && (ops[i].axis < 0 || ops[i].axis >= ndim_)) {
      throw InvalidArgument("detwin axis out of range");
    }
  }
  const int iters = recipe_iterations(ops, count);
  const std::size_t needed = static_cast<std::size_t>(std::max(iters, 1)) * starts_;
  trace("run: %d iterations, errs %zu -> %zu", iters, errs_.size(), needed);
  if (errs_.size() < needed) errs_ = DeviceBuffer<double>(needed);
  capacity_ = iters;
  const Ctrl ctrl{errs_.get(), capacity_, 0.0f, 0.0f, counters_.get()};
  set_ctrl(ctrl_.get(), ctrl, stream_);
  QPB_CHECK(cudaMemsetAsync(errs_.get(), 0, needed * sizeof(double), stream_));
  QPB_CHECK(cudaMemsetAsync(counters_.get(), 0, groups_ * sizeof(int), stream_));
  stream_.sync();
  run_iterations_ = 0;
}

void Solver::apply(const OpDesc& o) {
  switch (o.kind) {
    case kOpShrinkwrap:
      shrinkwrap(o);
      break;
    case kOpDetwinBegin:
      detwin_begin(o.axis);
      break;
    case kOpDetwinEnd:
      detwin_end();
      break;
    default:
      throw std::logic_error("Solver::apply: not a support operation");
  }
}

void Solver::end_run() {
  collect_errors(run_iterations_);
  check_waits(plans_, stream_);
}

void Solver::require_fp16_passes() const {
  struct Need {
    Mode mode;
    int axis3;
  };
  std::vector<Need> needs{{Mode::kMod, runner_.outer()}, {Mode::kUpd, 2}, {Mode::kFwdFromX, 2}};
  if (runner_.has_mid()) {
    needs.push_back({Mode::kInv, 1});
    needs.push_back({Mode::kFwd, 1});
  }
  for (const Need& need : needs) {
    // every launch size the solver uses: one group, and all starts at once
    for (int count : {batch_, starts_}) {
      PassParams p = runner_.params(need.mode, need.axis3, count);
      p.wave_half = 1;
      p.iter_half = options_.variant == Variant::kHalf ? 1 : 0;
      p.amp_tiled = need.mode == Mode::kMod ? kAmpTiledLines : 0;
      const bool column = column_pass_lines(p, need.mode) > 0;
      p.amp_tiled = need.mode == Mode::kMod && p.S > 1 ? kAmpTiledElements : 0;
      if (!column && !(fast_passes_enabled() && fast_pass_supports(p))) {
        throw InvalidArgument("the half and mixed variants need the register-resident or column "
                              "pass on every axis; this shape and start grouping have none on axis " +
                              std::to_string(need.axis3 - (3 - ndim_)));
      }
    }
  }
}

void Solver::set_wait(int tries, bool starve) {
  if (tries < 1) throw InvalidArgument("the wait limit must be >= 1 poll");
  stream_.sync();
  graphs_.clear();
  runner_.set_wait(tries, starve);
}

const char* op_name(int kind) {
  switch (kind) {
    case kOpER: return "ER";
    case kOpHIO: return "HIO";
    case kOpRAAR: return "RAAR";
    case kOpShrinkwrap: return "Shrinkwrap";
    case kOpDetwinBegin: return "DetwinBegin";
    case kOpDetwinEnd: return "DetwinEnd";
    default: return "op";
  }
}

void Solver::run(const OpDesc* ops, std::size_t count) {
  const NvtxRange recipe_range("recipe", recipe_iterations(ops, count));
  begin_run(ops, count);
  for (std::size_t i = 0; i < count; ++i) {
    const OpDesc& o = ops[i];
    trace("run op %zu/%zu kind=%d n=%d (iteration %d)", i, count, o.kind, o.n, iteration_);
    const NvtxRange stage_range(op_name(o.kind), o.n);
    switch (o.kind) {
      case kOpER:
        iterate(o.n, er_coefficients());
        break;
      case kOpHIO:
        iterate(o.n, hio_coefficients(o.beta));
        break;
      case kOpRAAR:
        iterate(o.n, raar_coefficients(o.beta));
        break;
      default:
        apply(o);
        break;
    }
  }
  end_run();
}

void Solver::begin_iterate(Coefficients c) {
  if (options_.variant == Variant::kMixed) {
    // The mixed variant's fp16 wave serves HIO and RAAR; ER (coefficients
    // 0, 0) runs entirely in FP32 (the reference's src/cuda/cuda_solver.cu
    // mixed path), so a stage boundary may change the wave's storage.
    const bool half = !(c.a == 0.0f && c.b == 0.0f);
    if (half != wave_half_) {
      wave_half_ = half;
      wave_valid_ = false;
    }
  }
  if (!wave_valid_) establish_wave();
  set_coefficients(ctrl_.get(), c.a, c.b, stream_);
}

int Solver::chunk_length(int remaining) const {
  const int every = options_.sync_every;
  return std::min(remaining, every - iteration_ % every);
}

void Solver::prepare_branches() {
  if (groups_ > 1 && branches_.empty() && batched() && !resident_) {
    // one branch stream per group plus a fork event and a join event per group
    for (int g = 0; g < groups_; ++g) branches_.push_back(std::make_unique<Stream>());
    branch_events_.resize(static_cast<std::size_t>(groups_) + 1);
    for (auto& e : branch_events_) QPB_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
}

// `len` iterations of every start, enqueued on `s` (captured into a graph by
// the batched variant): the resident kernel, or the groups' passes, each group
// a parallel branch so that one group's modulus pass can overlap another
// group's update pass; the plain variant runs groups one after another.
void Solver::enqueue_chunk_body(int len, cudaStream_t s) {
  if (resident_) {
    enqueue_chunk(len, s);
  } else if (persistent_) {
    QPB_CHECK(cudaMemsetAsync(work_.get(), 0, work_.size() * sizeof(unsigned), s));
    const int outer = runner_.outer();
    launch_persistent(base(Mode::kMod, outer, 0), base(Mode::kUpd, 2, 0), starts_, len,
                      work_.get(), s);
  } else if (groups_ > 1 && batched()) {
    if (branches_.empty()) throw std::logic_error("prepare_branches() was not called");
    QPB_CHECK(cudaEventRecord(branch_events_[0], s));
    for (int g = 0; g < groups_; ++g) {
      cudaStream_t b = *branches_[g];
      QPB_CHECK(cudaStreamWaitEvent(b, branch_events_[0], 0));
      for (int i = 0; i < len; ++i) enqueue_iteration(g, b);
      QPB_CHECK(cudaEventRecord(branch_events_[g + 1], b));
      QPB_CHECK(cudaStreamWaitEvent(s, branch_events_[g + 1], 0));
    }
  } else {
    for (int g = 0; g < groups_; ++g) {
      for (int i = 0; i < len; ++i) enqueue_iteration(g, s);
    }
  }
}

void Solver::end_chunk(int len) {
  iteration_ += len;
  run_iterations_ += len;
  if (progress_ && iteration_ % options_.sync_every == 0) report();
}

void Solver::iterate(int count, Coefficients c) {
  begin_iterate(c);
  for (int done = 0; done < count;) {
    const int len = chunk_length(count - done);
    if (batched()) {
      // graphs by chunk length and wave storage (the mixed variant switches it)
      const int key = 2 * len + (wave_half_ ? 1 : 0);
      auto it = graphs_.find(key);
      trace("iterate chunk len=%d graph=%s", len, it == graphs_.end() ? "capture" : "cached");
      if (it == graphs_.end()) {
        prepare_branches();
        const unsigned long long before = launches();
        QPB_CHECK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        try {
          enqueue_chunk_body(len, stream_);
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
      enqueue_chunk_body(len, stream_);
    }
    end_chunk(len);
    done += len;
  }
}

int Solver::profile_passes(int iterations, double* ms) {
  if (iterations < 1) throw InvalidArgument("iterations must be >= 1");
  if (!wave_valid_) establish_wave();
  // The solver's state is left as it was. The timed passes run against a
  // control block of their own (no error rows, ER coefficients, iteration
  // counters of their own), and the iterate and the wave are copied aside and
  // copied back afterwards: outside the modulus pass the transforms are
  // unnormalised, so one pass repeated on its own scales the arrays (by n^2
  // for four inverse transforms of n points) until they overflow.
  const std::size_t xb = x_.size() * sizeof(float2);
  const std::size_t hb = xh_.size() * sizeof(std::uint32_t);
  const std::size_t wb = w_.size() * sizeof(float2);
  DeviceBuffer<unsigned char> kept(xb + hb + wb);
  struct Span {
    unsigned char* live;
    unsigned char* kept;
    std::size_t bytes;
  };
  const std::array<Span, 3> spans{{{reinterpret_cast<unsigned char*>(x_.get()), kept.get(), xb},
                                   {reinterpret_cast<unsigned char*>(xh_.get()), kept.get() + xb, hb},
                                   {reinterpret_cast<unsigned char*>(w_.get()), kept.get() + xb + hb, wb}}};
  for (const Span& sp : spans) {
    if (sp.bytes) {
      QPB_CHECK(cudaMemcpyAsync(sp.kept, sp.live, sp.bytes, cudaMemcpyDeviceToDevice, stream_));
    }
  }
  struct PutBack {
    const std::array<Span, 3>& spans;
    cudaStream_t stream;
    ~PutBack() {
      for (const Span& sp : spans) {
        if (sp.bytes) cudaMemcpyAsync(sp.live, sp.kept, sp.bytes, cudaMemcpyDeviceToDevice, stream);
      }
      cudaStreamSynchronize(stream);  // before `kept` is freed
    }
  };
  const PutBack put_back{spans, stream_};
  DeviceBuffer<Ctrl> own_ctrl(1);
  DeviceBuffer<int> own_counters(static_cast<std::size_t>(groups_));
  QPB_CHECK(cudaMemsetAsync(own_counters.get(), 0, sizeof(int) * groups_, stream_));
  set_ctrl(own_ctrl.get(), Ctrl{nullptr, 0, 0.0f, 0.0f, own_counters.get()}, stream_);
  struct SwapBack {
    DeviceBuffer<Ctrl>& a;
    DeviceBuffer<Ctrl>& b;
    ~SwapBack() { std::swap(a, b); }
  };
  std::swap(ctrl_, own_ctrl);
  const SwapBack swap_back{ctrl_, own_ctrl};
  if (resident_ || persistent_) {
    // One launch of `iterations` iterations between two events.
    cudaEvent_t e0{}, e1{};
    QPB_CHECK(cudaEventCreate(&e0));
    QPB_CHECK(cudaEventCreate(&e1));
    QPB_CHECK(cudaEventRecord(e0, stream_));
    enqueue_chunk_body(iterations, stream_);
    QPB_CHECK(cudaEventRecord(e1, stream_));
    stream_.sync();
    float t = 0.0f;
    QPB_CHECK(cudaEventElapsedTime(&t, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ms[0] = static_cast<double>(t) / iterations;
    return 1;
  }
  const int outer = runner_.outer();
  struct PassRef {
    Mode mode;
    int axis3;
  };
  std::vector<PassRef> passes{{Mode::kMod, outer}};
  if (runner_.has_mid()) passes.push_back({Mode::kInv, 1});
  passes.push_back({Mode::kUpd, 2});
  if (runner_.has_mid()) passes.push_back({Mode::kFwd, 1});
  const int np = static_cast<int>(passes.size());
  std::vector<cudaEvent_t> events(static_cast<std::size_t>(2 * np));
  for (auto& e : events) QPB_CHECK(cudaEventCreate(&e));
  // Each pass runs `iterations` times back to back from one captured graph
  // (replayed once untimed, then once between two events), so the host's
  // launch cost stays out of the figure and the mean is the pass's device time
  // per launch (the next launch of the same pass follows at the device's own
  // launch spacing).
  for (int p = 0; p < np; ++p) {
    const unsigned long long before = launches();
    QPB_CHECK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try {
      for (int it = 0; it < iterations; ++it) {
        for (int g = 0; g < groups_; ++g) {
          runner_.launch(passes[p].mode, passes[p].axis3,
                         base(passes[p].mode, passes[p].axis3, g), stream_);
        }
      }
    } catch (...) {
      cudaGraph_t broken{};
      cudaStreamEndCapture(stream_, &broken);
      if (broken) cudaGraphDestroy(broken);
      for (auto& e : events) cudaEventDestroy(e);
      throw;
    }
    cudaGraph_t captured{};
    QPB_CHECK(cudaStreamEndCapture(stream_, &captured));
    const unsigned long long kernels = launches() - before;
    count_launches(0ULL - kernels);  // counted on every replay instead
    const Graph graph(captured, kernels);
    graph.launch(stream_);
    QPB_CHECK(cudaEventRecord(events[2 * p], stream_));
    graph.launch(stream_);
    QPB_CHECK(cudaEventRecord(events[2 * p + 1], stream_));
    stream_.sync();
  }
  for (int p = 0; p < np; ++p) {
    float t = 0.0f;
    QPB_CHECK(cudaEventElapsedTime(&t, events[2 * p], events[2 * p + 1]));
    ms[p] = static_cast<double>(t) / iterations;
  }
  for (auto& e : events) cudaEventDestroy(e);
  return np;
}

void Solver::shrinkwrap(const OpDesc& o) {
  // Blur |x| with exp(-2 (pi sigma f)^2) one axis at a time, reduce the level
  // in the last pass, threshold (kernels.cpp:77-102).
  const float half_pi = kTwoPi / 2;
  const float k = -2.0f * half_pi * half_pi * o.sigma * o.sigma;
  const int outer = runner_.outer();
  // A batched solver blurs every start in one launch per axis (one level
  // accumulator per start), whatever its start groups; the plain variant
  // keeps one start per launch like the rest of its iteration.
  const bool together = batched();
  const int chunks = together ? 1 : groups_;
  const int count = together ? starts_ : batch_;
  auto params = [&](Mode mode, int axis3, int g) {
    PassParams p = base(mode, axis3, g);
    p.lines = runner_.params(mode, axis3, count).lines;
    p.blur_k = k;
    return p;
  };
  // The blur runs in a complex64 wave whatever the wave's storage (an fp16
  // iterate is widened as it is read); the wave is re-established afterwards.
  const bool wave_half = wave_half_;
  wave_half_ = false;
  for (int g = 0; g < chunks; ++g) {
    QPB_CHECK(cudaMemsetAsync(level_.get(), 0, count * sizeof(LevelAcc), stream_));
    runner_.launch(Mode::kBlurMag, outer, params(Mode::kBlurMag, outer, g), stream_);
    if (runner_.has_mid()) runner_.launch(Mode::kBlur, 1, params(Mode::kBlur, 1, g), stream_);
    PassParams last = params(Mode::kBlur, 2, g);
    last.level_method = o.method + 1;
    runner_.launch(Mode::kBlur, 2, last, stream_);
    shrinkwrap_threshold(w(g), level_.get(), n_, count, o.method + 1, o.threshold, support(g),
                         stream_);
  }
  wave_half_ = wave_half;
  wave_valid_ = false;
}

void Solver::detwin_begin(int axis) {
  const std::size_t total = static_cast<std::size_t>(starts_) * n_;
  QPB_CHECK(cudaMemcpyAsync(saved_.get(), support_.get(), total, cudaMemcpyDeviceToDevice, stream_));
  detwin(support_.get(), moments_.get(), d_, axis + (3 - ndim_), starts_, stream_);
}

void Solver::detwin_end() {
  const std::size_t total = static_cast<std::size_t>(starts_) * n_;
  QPB_CHECK(cudaMemcpyAsync(support_.get(), saved_.get(), total, cudaMemcpyDeviceToDevice, stream_));
}

float Solver::to_error(double num, int start) const {
  return static_cast<float>(std::sqrt(num / (energies_[start / spp_] + kEps)));
}

void Solver::collect_errors(int iterations) {
  trace("collect_errors iterations=%d starts=%d", iterations, starts_);
  host_errs_.resize(static_cast<std::size_t>(std::max(iterations, 1)) * starts_);
  if (iterations > 0) {
    QPB_CHECK(cudaMemcpyAsync(host_errs_.data(), errs_.get(),
                              static_cast<std::size_t>(iterations) * starts_ * sizeof(double),
                              cudaMemcpyDeviceToHost, stream_));
  }
  stream_.sync();
  for (int t = 0; t < iterations; ++t) {
    for (int s = 0; s < starts_; ++s) {
      errors_[s].push_back(to_error(host_errs_[static_cast<std::size_t>(t) * starts_ + s], s));
    }
  }
}

std::vector<float> Solver::latest_errors() {
  if (run_iterations_ < 1) throw std::logic_error("latest_errors before any iteration");
  std::vector<double> row(static_cast<std::size_t>(starts_));
  QPB_CHECK(cudaMemcpyAsync(row.data(),
                            errs_.get() + static_cast<std::size_t>(run_iterations_ - 1) * starts_,
                            row.size() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  stream_.sync();
  std::vector<float> latest(row.size());
  for (std::size_t s = 0; s < row.size(); ++s) latest[s] = to_error(row[s], static_cast<int>(s));
  return latest;
}

void Solver::report() {
  const std::vector<float> latest = latest_errors();
  progress_(progress_user_, iteration_, latest.data(), starts_);
}

void Solver::iterate_f32(float2* out) {
  const std::size_t total = static_cast<std::size_t>(starts_) * n_;
  if (iter_half_) from_half(xh_.get(), x_.get(), static_cast<long long>(total), stream_);
  roll<float2>(x_.get(), out, d_, starts_, false, stream_);
  if (fp16_wave_variant()) {
    const std::size_t block = static_cast<std::size_t>(spp_) * n_;
    for (int q = 0; q < problems_; ++q) {
      scale_complex(out + q * block, static_cast<long long>(block),
                    amp_scale_[static_cast<std::size_t>(q)], stream_);
    }
  }
}

void Solver::results_device(float2* objects, std::uint8_t* supports, float* errors) {
  if (objects) iterate_f32(objects);
  if (supports) roll<std::uint8_t>(support_.get(), supports, d_, starts_, false, stream_);
  stream_.sync();
  if (errors) {
    const std::size_t count = error_count();
    for (int s = 0; s < starts_; ++s) {
      std::copy(errors_[s].begin(), errors_[s].end(), errors + static_cast<std::size_t>(s) * count);
    }
  }
}

void Solver::results(float2* objects, std::uint8_t* supports, float* errors) {
  const std::size_t block = static_cast<std::size_t>(spp_) * n_;
  const std::size_t count = error_count();
  std::vector<float2*> o(static_cast<std::size_t>(problems_), nullptr);
  std::vector<std::uint8_t*> s(o.size(), nullptr);
  std::vector<float*> e(o.size(), nullptr);
  for (std::size_t q = 0; q < o.size(); ++q) {
    if (objects) o[q] = objects + q * block;
    if (supports) s[q] = supports + q * block;
    if (errors) e[q] = errors + q * spp_ * count;
  }
  results_per_problem(o.data(), s.data(), e.data());
}

void Solver::results_per_problem(float2* const* objects, std::uint8_t* const* supports,
                                 float* const* errors) {
  // centre-origin copies on the device, then one transfer per problem
  // straight into the caller's memory
  const std::size_t block = static_cast<std::size_t>(spp_) * n_;
  if (objects) {
    iterate_f32(w_.get());
    wave_valid_ = false;
    for (int q = 0; q < problems_; ++q) {
      if (!objects[q]) continue;
      QPB_CHECK(cudaMemcpyAsync(objects[q], w_.get() + q * block, block * sizeof(float2),
                                cudaMemcpyDeviceToHost, stream_));
    }
  }
  if (supports) {
    roll<std::uint8_t>(support_.get(), saved_.get(), d_, starts_, false, stream_);
    for (int q = 0; q < problems_; ++q) {
      if (!supports[q]) continue;
      QPB_CHECK(cudaMemcpyAsync(supports[q], saved_.get() + q * block, block,
                                cudaMemcpyDeviceToHost, stream_));
    }
  }
  stream_.sync();
  if (errors) {
    const std::size_t count = error_count();
    for (int q = 0; q < problems_; ++q) {
      if (!errors[q]) continue;
      for (int j = 0; j < spp_; ++j) {
        const auto& row = errors_[static_cast<std::size_t>(q) * spp_ + j];
        std::copy(row.begin(), row.end(), errors[q] + static_cast<std::size_t>(j) * count);
      }
    }
  }
}

// ------------------------------------------------------------------- operators
// Line plans (device twiddle tables) of the single operators and the problem
// set-up, kept per device for the process so that repeated calls allocate
// nothing for them.
PlanCache& operator_plans() {
  static std::mutex mutex;
  static std::map<int, std::unique_ptr<PlanCache>> per_device;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  auto& slot = per_device[device];
  if (!slot) slot = std::make_unique<PlanCache>();
  return *slot;
}

namespace {

struct OperatorContext {
  Dims3 d;
  int ndim;
  PlanCache& plans;
  Stream stream;
  PassRunner runner;
  OperatorContext(Dims3 dims, int nd)
      : d(dims), ndim(nd), plans(operator_plans()), runner(dims, nd, plans) {}
};

ProblemView view_of(int ndim, const long long* shape) {
  ProblemView v;
  v.ndim = ndim;
  if (ndim != 2 && ndim != 3) throw InvalidArgument("shape must be 2D or 3D, got ndim=" + std::to_string(ndim));
  for (int a = 0; a < ndim; ++a) v.shape[a] = shape[a];
  return v;
}

}  // namespace

float modulus_project(const ProblemView& problem, float2* obj, AmpStorage storage) {
  const Dims3 d = dims_of(problem);
  const long long n = d.n();
  OperatorContext ctx(d, problem.ndim);
  const auto amp = host_roll(problem.amplitude, d, true);
  std::vector<std::uint8_t> mask(static_cast<std::size_t>(n), 0);
  if (problem.mask) {
    mask = host_roll(problem.mask, d, true);
    for (auto& m : mask) m = m != 0;
  }
  const double energy = usable_energy(amp, mask);
  auto d_amp = upload(signed_amplitude(amp, mask, storage), ctx.stream);
  auto d_x = upload(host_roll(obj, d, true), ctx.stream);
  DeviceBuffer<float2> d_w(static_cast<std::size_t>(n));
  DeviceBuffer<double> errs(1);
  DeviceBuffer<int> counter(1);
  DeviceBuffer<Ctrl> ctrl(1);
  QPB_CHECK(cudaMemsetAsync(errs.get(), 0, sizeof(double), ctx.stream));
  QPB_CHECK(cudaMemsetAsync(counter.get(), 0, sizeof(int), ctx.stream));
  const Ctrl c{errs.get(), 1, 0.0f, 0.0f, counter.get()};
  set_ctrl(ctrl.get(), c, ctx.stream);
  auto params = [&](Mode m, int axis3) {
    PassParams p = ctx.runner.params(m, axis3, 1);
    p.w = d_w.get();
    p.x = d_x.get();
    p.amp = d_amp.get();
    p.ctrl = ctrl.get();
    p.starts_total = 1;
    p.amp_storage = storage;
    return p;
  };
  const int outer = ctx.runner.outer();
  ctx.runner.launch(Mode::kFwdFromX, 2, params(Mode::kFwdFromX, 2), ctx.stream);
  if (ctx.runner.has_mid()) ctx.runner.launch(Mode::kFwd, 1, params(Mode::kFwd, 1), ctx.stream);
  ctx.runner.launch(Mode::kMod, outer, params(Mode::kMod, outer), ctx.stream);
  if (ctx.runner.has_mid()) ctx.runner.launch(Mode::kInv, 1, params(Mode::kInv, 1), ctx.stream);
  ctx.runner.launch(Mode::kInv, 2, params(Mode::kInv, 2), ctx.stream);
  std::vector<float2> host(static_cast<std::size_t>(n));
  double num = 0.0;
  QPB_CHECK(cudaMemcpyAsync(host.data(), d_w.get(), host.size() * sizeof(float2),
                            cudaMemcpyDeviceToHost, ctx.stream));
  QPB_CHECK(cudaMemcpyAsync(&num, errs.get(), sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
  ctx.stream.sync();
  check_waits(ctx.plans, ctx.stream);
  const auto centred = host_roll(host.data(), d, false);
  std::copy(centred.begin(), centred.end(), obj);
  return static_cast<float>(std::sqrt(num / (energy + kEps)));
}

void support_project_host(const std::uint8_t* support, float2* obj, long long count) {
  Stream s;
  DeviceBuffer<float2> x(static_cast<std::size_t>(count));
  DeviceBuffer<std::uint8_t> sup(static_cast<std::size_t>(count));
  QPB_CHECK(cudaMemcpyAsync(x.get(), obj, count * sizeof(float2), cudaMemcpyHostToDevice, s));
  QPB_CHECK(cudaMemcpyAsync(sup.get(), support, count, cudaMemcpyHostToDevice, s));
  support_project(x.get(), sup.get(), count, 1, s);
  QPB_CHECK(cudaMemcpyAsync(obj, x.get(), count * sizeof(float2), cudaMemcpyDeviceToHost, s));
  s.sync();
}

void gaussian_blur(const float* image, int ndim, const long long* shape, float sigma, float* out) {
  const Dims3 d = dims_of(view_of(ndim, shape));
  if (!(sigma >= 0.0f)) throw InvalidArgument("sigma must be >= 0");
  const long long n = d.n();
  OperatorContext ctx(d, ndim);
  // A circular blur commutes with the fftshift roll (operators.cpp:33-39).
  std::vector<float2> host(static_cast<std::size_t>(n));
  for (long long i = 0; i < n; ++i) host[i] = {image[i], 0.0f};
  auto w = upload(host, ctx.stream);
  const float half_pi = kTwoPi / 2;
  const float k = -2.0f * half_pi * half_pi * sigma * sigma;
  for (int axis3 = ctx.runner.outer(); axis3 < 3; ++axis3) {
    PassParams p = ctx.runner.params(Mode::kBlur, axis3, 1);
    p.w = w.get();
    p.blur_k = k;
    ctx.runner.launch(Mode::kBlur, axis3, p, ctx.stream);
  }
  QPB_CHECK(cudaMemcpyAsync(host.data(), w.get(), host.size() * sizeof(float2),
                            cudaMemcpyDeviceToHost, ctx.stream));
  ctx.stream.sync();
  check_waits(ctx.plans, ctx.stream);
  for (long long i = 0; i < n; ++i) out[i] = host[i].x;
}

void half_support(const std::uint8_t* support, int ndim, const long long* shape, int axis,
                  std::uint8_t* out) {
  const Dims3 d = dims_of(view_of(ndim, shape));
  if (axis < 0 || axis >= ndim) throw InvalidArgument("detwin axis out of range");
  const long long n = d.n();
  Stream s;
  auto ordered = host_roll(support, d, true);
  for (auto& v : ordered) v = v != 0;
  auto dev = upload(ordered, s);
  DeviceBuffer<unsigned long long> moments(2);
  detwin(dev.get(), moments.get(), d, axis + (3 - ndim), 1, s);
  QPB_CHECK(cudaMemcpyAsync(ordered.data(), dev.get(), static_cast<std::size_t>(n),
                            cudaMemcpyDeviceToHost, s));
  s.sync();
  const auto centred = host_roll(ordered.data(), d, false);
  std::copy(centred.begin(), centred.end(), out);
}

}  // namespace qpb
