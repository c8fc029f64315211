/* qpb.h -- C ABI of the B200 phase-retrieval backend (libqpb.so).
 *
 * The backend is a new implementation of QoraPhaseCU's qpcu::Solver
 * (include/qoraphasecu/solver.hpp:67-74 in the reference), selected by a new
 * qpcu::Backend value. Everything crosses this boundary as plain pointers and
 * sizes; no C++ exception crosses it. Every function returns a qpb_status;
 * qpb_last_error() gives the message of the last failure on the calling thread.
 *
 * Arrays are centre-origin (index n/2 along each axis is q = 0 or r = 0), as in
 * the reference's public API (include/qoraphasecu/problem.hpp:24-31). Complex
 * arrays are interleaved complex64 (re, im float pairs).
 */
#ifndef QPB_H_
#define QPB_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define QPB_API __attribute__((visibility("default")))
#else
#define QPB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. QPB_INVALID_ARGUMENT is the reference's std::invalid_argument
 * (src/core/solver.cpp:62-78, recipe.cpp:30-61, problem.cpp:21-56);
 * QPB_RUNTIME_ERROR its std::runtime_error (src/cuda/common.cuh:15-31). */
typedef enum qpb_status {
  QPB_OK = 0,
  QPB_INVALID_ARGUMENT = 1,
  QPB_RUNTIME_ERROR = 2,
  QPB_TIMEOUT = 3
} qpb_status;

/* Storage type of the amplitude (FP32 arithmetic either way). */
typedef enum qpb_amp_storage { QPB_AMP_F32 = 0, QPB_AMP_F16 = 1, QPB_AMP_BF16 = 2 } qpb_amp_storage;

/* Execution schedule. BATCHED runs `batch` starts per launch with iterations
 * replayed from CUDA graphs; PLAIN runs one start per launch, launched
 * directly (the in-repo baseline). HALF and MIXED are BATCHED with fp16
 * storage, the reference's Variant::half and Variant::mixed
 * (src/cuda/half.cu:14-83, cuda_solver.cu:74-86): HALF stores the iterate and
 * the wave as fp16 pairs; MIXED stores the wave in fp16 during HIO and RAAR,
 * runs ER entirely in FP32 and keeps an FP32 iterate. Both divide the
 * amplitude by its peak (objects are returned in the data's scale), compute
 * in FP32, need power-of-two extents of 16..1024 and an FP32 amplitude, and run
 * the streamed schedule. Replaces qpcu::Variant (solver.hpp:21-29). */
typedef enum qpb_variant {
  QPB_VARIANT_BATCHED = 0,
  QPB_VARIANT_PLAIN = 1,
  QPB_VARIANT_HALF = 2,
  QPB_VARIANT_MIXED = 3
} qpb_variant;

/* How BATCHED iterations run (no counterpart in the reference). STREAMED: two
 * line passes per 2D iteration (four in 3D) through HBM, start groups as
 * parallel graph branches. RESIDENT: square 2D problems of side 64, 128 or 256
 * only; each start's iterate stays in the shared memory of a thread-block
 * cluster for a whole chunk of sync_every iterations, one launch per chunk.
 * PERSISTENT: 2D problems with sides of 64, 128 or 256 (complex64 storage);
 * a chunk of sync_every iterations of every start is one launch whose CTAs
 * claim the passes' tiles from a work list, each tile waiting (bounded) only
 * for the tiles of its own start that it reads, so the passes of different
 * starts overlap with no launch boundary. AUTO: the autotuner times the
 * candidates once per shape and start count. */
typedef enum qpb_schedule {
  QPB_SCHEDULE_AUTO = 0,
  QPB_SCHEDULE_STREAMED = 1,
  QPB_SCHEDULE_RESIDENT = 2,
  QPB_SCHEDULE_PERSISTENT = 3
} qpb_schedule;

/* A made problem: the fields of qpcu::Problem (problem.hpp:26-31). */
typedef struct qpb_problem {
  int ndim;                /* 2 or 3 */
  int64_t shape[3];        /* slowest axis first */
  const float* amplitude;  /* numel, sqrt(clip(intensity, 0)) */
  const uint8_t* mask;     /* numel, 1 = unusable pixel; NULL = every pixel usable */
  const uint8_t* support;  /* numel, 1 = inside the object */
} qpb_problem;

/* qpcu::Options (solver.hpp:40-55) minus the backend and progress fields. */
typedef struct qpb_options {
  int starts;              /* >= 1 */
  int batch;               /* starts per launch, must divide starts; 0 = all */
  uint64_t seed;           /* seed of the random starting phases */
  const float* start;      /* starts * numel complex64 centre-origin objects, or NULL */
  int sync_every;          /* iterations per graph launch and progress interval, >= 1 */
  int variant;             /* qpb_variant */
  int amp_storage;         /* qpb_amp_storage */
  int device;              /* CUDA device ordinal; -1 = the calling thread's current device */
  void* stream;            /* cudaStream_t the solver enqueues on; NULL = a stream of its own */
  int schedule;            /* a qpb_schedule value; used by BATCHED only */
} qpb_options;

/* One recipe operation: the POD form of qpcu::Op (recipe.hpp:44), the same
 * seven fields as the reference's Python op tuple (python/bindings.cpp:22-23). */
typedef enum qpb_op_kind {
  QPB_OP_ER = 0,
  QPB_OP_HIO = 1,
  QPB_OP_RAAR = 2,
  QPB_OP_SHRINKWRAP = 3,
  QPB_OP_DETWIN_BEGIN = 4,
  QPB_OP_DETWIN_END = 5
} qpb_op_kind;

typedef struct qpb_op {
  int kind;        /* qpb_op_kind */
  int n;           /* iterations (ER, HIO, RAAR) */
  float beta;      /* HIO, RAAR */
  float threshold; /* Shrinkwrap */
  float sigma;     /* Shrinkwrap */
  int method;      /* Shrinkwrap: 0 max, 1 rms (qpcu::Threshold, recipe.hpp:25) */
  int axis;        /* DetwinBegin */
} qpb_op;

typedef struct qpb_solver qpb_solver;

/* Called every sync_every iterations with the iteration count so far and the
 * latest Fourier error of each start (qpcu::Progress, solver.hpp:36-38). */
typedef void (*qpb_progress_fn)(void* user, int iteration, const float* errors, int count);

/* Message of the last failed call on this thread ("" if none). */
QPB_API const char* qpb_last_error(void);

/* 1 when a CUDA device is present (qpcu::cuda_available, solver.hpp:85). */
QPB_API int qpb_cuda_available(void);

/* Selects the device that calls without a solver (make_problem, the single
 * operators) use on the calling thread. No counterpart in the reference, which
 * always uses the current device (src/cuda/kernels.cu:15-24). */
QPB_API qpb_status qpb_set_device(int device);

/* Replaces qpcu::cuda_device_info (solver.hpp:87-98). name_out holds name_len bytes. */
QPB_API qpb_status qpb_device_info(char* name_out, size_t name_len, int* sm_major, int* sm_minor,
                           size_t* memory_bytes, size_t* l2_bytes, double* peak_bandwidth_gbs);

/* qpcu::make_problem (problem.hpp:35-37, problem.cpp:40-70): validates the
 * inputs, amplitude = sqrt(max(I, 0)); a NULL support is replaced by the
 * autocorrelation support at `support_threshold`. Outputs are numel each. */
QPB_API qpb_status qpb_make_problem(const float* intensity, int ndim, const int64_t* shape,
                            const uint8_t* support, const uint8_t* mask, float support_threshold,
                            float* amplitude_out, uint8_t* mask_out, uint8_t* support_out);

/* qpcu::autocorrelation_support (problem.hpp:42-43, problem.cpp:72-88). */
QPB_API qpb_status qpb_autocorrelation_support(const float* intensity, int ndim, const int64_t* shape,
                                       float threshold, uint8_t* out);

/* qpcu::half_support (problem.hpp:51-52, problem.cpp:101-127), on the device. */
QPB_API qpb_status qpb_half_support(const uint8_t* support, int ndim, const int64_t* shape, int axis,
                            uint8_t* out);

/* qpcu::make_solver for the new backend (solver.cpp:61-86 ->
 * detail::make_cuda_solver, backends.hpp:9-10): uploads the problem and draws
 * the starts. */
QPB_API qpb_status qpb_create(const qpb_problem* problem, const qpb_options* options, qpb_solver** out);

/* Device-resident inputs and outputs (no counterpart in the reference, whose
 * Python layer copies through numpy, python/bindings.cpp:37-41): callers that
 * hold their data in device memory (torch tensors, a detector pipeline's
 * buffers) set up, run and read a reconstruction without any array crossing to
 * the host.
 *   qpb_make_problem_device: qpb_make_problem on device arrays (centre-origin,
 * numel each; support and mask may be NULL), the autocorrelation support
 * computed on the device; enqueued on `stream` (a cudaStream_t, NULL = legacy
 * default stream), returns after it completes.
 *   qpb_create_device: qpb_create whose problem arrays are device pointers;
 * options->start, when given, is a device pointer too.
 *   qpb_results_device: qpb_results with objects (starts * numel complex64) and
 * supports (starts * numel) written to device memory; errors to host memory.
 * Problems of one shape only. */
QPB_API qpb_status qpb_make_problem_device(const float* intensity, int ndim, const int64_t* shape,
                                           const uint8_t* support, const uint8_t* mask,
                                           float support_threshold, float* amplitude_out,
                                           uint8_t* mask_out, uint8_t* support_out,
                                           void* stream);
QPB_API qpb_status qpb_create_device(const qpb_problem* problem, const qpb_options* options,
                                     qpb_solver** out);
QPB_API qpb_status qpb_results_device(qpb_solver* solver, float* objects, uint8_t* supports,
                                      float* errors);

/* Many problems, any mix of shapes, reconstructed together (no counterpart in
 * the reference, which builds one solver per problem). options->starts starts
 * per problem; options->start, when given, holds every problem's starts in
 * problem order. Problems of one shape share one batched solver (its schedule
 * autotuned for that shape and start count); every chunk of sync_every
 * iterations of every shape runs as ONE CUDA graph with the shapes as
 * parallel branches. qpb_run, qpb_results (problem order: problem q's block of
 * starts * numel(q) objects and supports, starts * error_count errors, blocks
 * back to back), qpb_starts (problems * starts) and qpb_destroy work on it;
 * qpb_profile_passes needs one shape. */
QPB_API qpb_status qpb_create_batch(const qpb_problem* problems, size_t n_problems,
                                    const qpb_options* options, qpb_solver** out);

/* qpcu::Solver::run (solver.hpp:72): validates and runs the recipe, continuing
 * from the current state; appends one error per iteration to every start. */
QPB_API qpb_status qpb_run(qpb_solver* solver, const qpb_op* ops, size_t n_ops);

/* Loads new problems into an existing solver (no counterpart in the reference):
 * the same number of problems as at creation, problem q in the shape problem q
 * had then (a batch of several shapes included), host or device arrays as at
 * creation; starts drawn from `seed` as a new solver would draw them, or given
 * in `start` (NULL = drawn; given device starts need one shape). Device
 * buffers, the schedule and the captured CUDA graphs are kept, so a caller
 * reconstructing a stream of same-shape patterns pays for allocation and graph
 * capture once. Error histories start afresh. */
QPB_API qpb_status qpb_reset(qpb_solver* solver, const qpb_problem* problems, size_t n_problems,
                             uint64_t seed, const float* start);

/* Bounded waits (no counterpart in the reference, whose kernels never wait on
 * one another). The line passes stage inputs by asynchronous bulk copies and
 * wait for them a bounded number of polls (about 4 million by default); a CTA
 * that gives up writes nothing and counts itself in a counter of the solver,
 * and the qpb_run that launched it returns QPB_TIMEOUT. `polls` sets the limit
 * for the launches that follow (captured graphs are re-captured). `starve`
 * non-zero is fault injection for tests of that path: the staged copies are
 * left out, so every staged wait runs out; results are invalid until the
 * solver is reset with starve 0 and qpb_reset. */
QPB_API qpb_status qpb_set_wait_limit(qpb_solver* solver, int polls, int starve);

/* Progress callback (Options::progress, solver.hpp:52-54); NULL disables it. */
QPB_API qpb_status qpb_set_progress(qpb_solver* solver, qpb_progress_fn fn, void* user);

/* Iterations run so far (the length of every start's error history). */
QPB_API qpb_status qpb_error_count(const qpb_solver* solver, size_t* count);
QPB_API qpb_status qpb_starts(const qpb_solver* solver, int* starts);

/* qpcu::Solver::results (solver.hpp:73) into caller buffers: objects
 * starts * numel complex64, supports starts * numel, errors starts * error_count.
 * Any output may be NULL. */
QPB_API qpb_status qpb_results(qpb_solver* solver, float* objects, uint8_t* supports, float* errors);

QPB_API void qpb_destroy(qpb_solver* solver);

/* Kernels this library has launched in this process; a replayed CUDA graph
 * counts each kernel node. No counterpart in the reference: it backs the
 * launch count that bench.py reports. */
QPB_API uint64_t qpb_kernel_launches(void);

/* Writes the autotuner's choices so far (one line per tuned shape and start
 * count: the starts per launch picked and the time of every candidate) into
 * `out` (NUL-terminated, at most `len` bytes). No counterpart in the reference,
 * which fixes the grouping through Options::batch (solver.hpp:44-46). */
QPB_API qpb_status qpb_tuning_report(char* out, size_t len);

/* Times each line pass of an iteration: pass p is launched `iterations` times
 * back to back (all start groups) from one captured CUDA graph, replayed once
 * untimed and once between two CUDA events on the solver's stream (the events
 * time the kernels, not the host's launch rate; the solver's stream must be
 * capturable, not the legacy default stream); ms_out[p] receives the mean time
 * per launch and
 * *n_passes their count (<= 8; 2D: modulus pass, update pass; 3D adds the
 * y-axis inverse and forward passes). With the resident schedule, *n_passes =
 * 1 and ms_out[0] is the mean time per iteration of one launch running all
 * `iterations`. Leaves the solver as it was: the passes run with ER
 * coefficients, write no error rows and count no iterations, and the iterate
 * and the wave are copied aside and back (one more copy of each on the device
 * during the call). No counterpart in the reference: it
 * feeds the per-kernel roofline that bench.py reports. */
QPB_API qpb_status qpb_profile_passes(qpb_solver* solver, int iterations, double* ms_out, int* n_passes);

/* The modulus projection of qpb_modulus_project for callers that must not
 * allocate device memory (no counterpart in the reference): applications that
 * reserve their whole GPU memory up front and may not grow it, and threads that
 * cannot afford cudaMalloc's implicit device synchronisation. It allocates
 * nothing; its scratch lives in one fixed __device__ array of the library.
 *   Every pointer except `shape` is device memory, arrays in FFT order (numpy
 * ifftshift of the centre-origin arrays): amplitude (numel float), mask (numel
 * uint8, NULL = all usable), x (numel complex64), out (numel complex64, may be
 * x), error_out (1 float: the Fourier error of x). Work is enqueued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) and the call
 * returns without waiting for it.
 *   Limits: at most 65536 elements and 4096 along any axis; larger shapes
 * return QPB_INVALID_ARGUMENT. The first call on a device looks up the array's
 * device address and configures kernels; make that first call before any
 * stream capture. All calls on a device share the array, which keeps the last
 * call's contents (each call clears what must start at zero; the twiddle
 * tables of the previous shape are reused): calls that overlap on the GPU,
 * e.g. on two streams, race on it.
 *   x and out must be 16-byte aligned (they are moved by bulk copies), the
 * amplitude and error_out 4-byte aligned; a misaligned pointer returns
 * QPB_INVALID_ARGUMENT before anything is launched. If a line pass gives up a
 * bounded wait for its staged inputs, *error_out is NaN and out is not the
 * projection. */
QPB_API qpb_status qpb_modulus_project_noalloc(int ndim, const int64_t* shape,
                                               const float* amplitude, const uint8_t* mask,
                                               const float* x, float* out, float* error_out,
                                               void* stream);

/* Amplitude loss and its gradient for gradient-based reconstruction (no
 * counterpart in the reference, whose solvers only project): for each of
 * `batch` objects x_b, loss[b] = sum over usable pixels of (|F x_b| - A)^2
 * with F the unitary FFT, and grad[b] = dL/dRe x_b + i dL/dIm x_b =
 * 2 F^H[(|y| - A) y / |y|] = 2 (x_b - P_M x_b) with the modulus projection of
 * qpb_modulus_project (src/cpu/kernels.cpp:25-42 in the reference).
 *   Device pointers, FFT order (numpy ifftshift of centre-origin arrays):
 * signed_amplitude (numel floats, the amplitude with -1 on masked pixels),
 * x and grad (batch * numel complex64, distinct), loss (batch doubles).
 * Enqueued on `stream` (cudaStream_t; NULL = legacy default stream); returns
 * without waiting. The first call per device and shape builds line plans
 * (device allocations kept for the process); calls on one device share a
 * control block, so calls that overlap on the GPU race. signed_amplitude, x
 * and grad must be 16-byte aligned (bulk copies move them), loss 8-byte
 * aligned; otherwise QPB_INVALID_ARGUMENT. If a line pass gives up a bounded
 * wait for its staged inputs, every loss is NaN. */
QPB_API qpb_status qpb_amplitude_loss_grad(int ndim, const int64_t* shape, int batch,
                                           const float* signed_amplitude, const float* x,
                                           float* grad, double* loss, void* stream);

/* The projection after a gradient step (no counterpart in the reference; it
 * follows qpb_support_project and adds a magnitude cap): for each of `batch`
 * objects of `numel` complex64 elements in x (device memory, in place), an
 * element outside the support (support[i] == 0; `support` is numel bytes of
 * device memory, shared by the objects) becomes 0, and one inside whose
 * magnitude exceeds `bound` is scaled onto the disc of radius `bound`; the
 * others are left unchanged. bound = +infinity applies the support alone.
 * Enqueued on `stream` (cudaStream_t; NULL = legacy default stream); returns
 * without waiting. x must be 8-byte aligned, bound > 0, batch in
 * [1, 65535]; otherwise QPB_INVALID_ARGUMENT. */
QPB_API qpb_status qpb_project_support_bound(int64_t numel, int batch, const uint8_t* support,
                                             float bound, float* x, void* stream);

/* qpcu::aligned_error (include/qoraphasecu/metrics.hpp:12, src/core/metrics.cpp:17-86)
 * for `batch` candidates at once, on the device: out[b] = ||a_b - ref|| / ||ref||
 * after the best integer translation (cross-correlation peak), global phase and
 * twin (conj(a(-r))). a: batch * numel complex64, reference: numel complex64,
 * out: batch floats; host arrays. */
QPB_API qpb_status qpb_aligned_error(const float* a, const float* reference, int ndim,
                                     const int64_t* shape, int batch, float* out);

/* Ensemble alignment and averaging (no counterpart in the reference, whose
 * README.md:222-224 leaves it to the user): the alignment of qpb_aligned_error
 * applied. errors: batch floats as qpb_aligned_error (may be NULL); aligned:
 * batch * numel complex64, object b -- or its twin, whichever fits better --
 * translated and phase-rotated onto the reference (may be NULL); mean: numel
 * complex64, the average of the aligned objects (may be NULL). Host arrays. */
QPB_API qpb_status qpb_align(const float* a, const float* reference, int ndim, const int64_t* shape,
                             int batch, float* errors, float* aligned, float* mean);

/* qpcu::simulate_intensity (problem.hpp:42, problem.cpp:90-99): |centred unitary
 * FFT(object)|^2 of a centre-origin complex64 object, the transform on the
 * device. Host arrays of numel elements. */
QPB_API qpb_status qpb_simulate_intensity(const float* object, int ndim, const int64_t* shape,
                                          float* out);

/* Single operators on centre-origin arrays (qpcu::cuda::, operators.hpp:25-33). */
QPB_API qpb_status qpb_modulus_project(const qpb_problem* problem, float* obj, int amp_storage,
                               float* error_out);
QPB_API qpb_status qpb_support_project(const uint8_t* support, float* obj, size_t count);
QPB_API qpb_status qpb_gaussian_blur(const float* image, int ndim, const int64_t* shape, float sigma,
                             float* out);

#ifdef __cplusplus
}
#endif

#endif /* QPB_H_ */
